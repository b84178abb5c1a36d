"""fs2_b200: fs2's particle-mesh / COLA time step and 2LPT initial conditions
on NVIDIA B200 (sm_100a).

* ``fs2_b200.fs`` -- drop-in for the reference's Python package ``fs``
  (fs.pm, fs.cola, fs.lpt, fs.Particles, fs.PowerSpectrum, fs.cosmology,
  fs.FFT), backed by the CPython extension ``fs._fs`` and libfs2gpu.so.
* ``include/fs2gpu.h`` -- the C ABI of libfs2gpu.so.
"""
import os

LIB_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib")
LIB_PATH = os.path.join(LIB_DIR, "libfs2gpu.so")
