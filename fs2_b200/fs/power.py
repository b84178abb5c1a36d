"""Linear power spectrum table (py/fs/power.py).

    ps = fs.PowerSpectrum('matterpower.dat')
    len(ps)  # number of rows
    ps[i]    # (k, P) of row i
"""
from . import _fs as c


class PowerSpectrum:
    """A tabulated `k P(k)` text file (CAMB matterpower.dat layout), read as
    the reference reads it; P(k) between rows is a natural cubic spline in
    log k - log P.

    Raises:
        IOError: if the file cannot be read.
    """

    def __init__(self, filename):
        self._ps = c._power_alloc(filename)

    def __len__(self):
        return c._power_n(self._ps)

    def __getitem__(self, i):
        """(k, P) of row i; IndexError outside the table."""
        return c._power_i(self._ps, i)

    def P(self, k):
        """The interpolated P(k)."""
        return c._power_P(self._ps, k)

    def sigma(self, R):
        """rms of the linear field smoothed with a top-hat of radius R."""
        return c._power_sigma(self._ps, R)
