"""fs -- fs2's Python API on a B200.

Same modules and names as the reference package (py/fs/__init__.py):
``fs.cosmology``, ``fs.lpt``, ``fs.pm``, ``fs.cola``, ``fs.msg``,
``fs.comm``, ``fs.leapfrog``, ``fs.Particles``, ``fs.PowerSpectrum``, ``fs.FFT``.  Importing
it does not start MPI (the reference calls MPI_Init here,
py/fs/__init__.py:17-19): one process drives one GPU.

The work is done by the CPython extension ``fs._fs`` (C++), which calls the
C ABI of libfs2gpu.so (include/fs2gpu.h).  If the extension was not built,
importing this package fails loudly rather than falling back to the CPU.
"""
import atexit

from . import _fs
from . import comm
from . import cosmology
from . import lpt
from . import pm
from . import cola
from . import leapfrog
from . import msg
from .particles import Particles
from .power import PowerSpectrum
from .fft import FFT

config_precision = _fs.config_precision

_fs.comm_mpi_init()
atexit.register(_fs.comm_mpi_finalise)
