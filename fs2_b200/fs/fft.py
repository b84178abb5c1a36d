"""3-D real mesh handle (py/fs/fft.py)."""
from . import _fs as c


class FFT:
    """A 3-D mesh in real or Fourier space.

    FFT(nc) allocates a new nc^3 mesh on the GPU; FFT(_fft) wraps a capsule
    returned by the library (the PM density mesh).
    """

    def __init__(self, arg):
        if isinstance(arg, int):
            self._fft = c._fft_alloc(arg)
        else:
            self._fft = arg

    def set_test_data(self):
        """Sets grid(ix, iy, iz) = (ix*nc + iy)*nc + iz + 1."""
        c._fft_set_test_data(self._fft)

    def asarray(self):
        """The real mesh as an (nc, nc, nc) float32 np.array."""
        return c._fft_fx_global_as_array(self._fft)
