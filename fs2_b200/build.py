"""Build the in-tree native parts of fs2_b200.

* fs2_b200/lib/libfs2gpu.so -- the CUDA library behind include/fs2gpu.h,
  compiled for sm_100a only (nvcc -gencode arch=compute_100a,code=sm_100a);
* fs2_b200/fs/_fs*.so -- the CPython extension fs._fs (C++), the drop-in
  for the reference's py/py_package.cpp method table, linked to the above.

Objects are rebuilt when a source or header is newer than the target.
Usage: python -m fs2_b200.build [--force]
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
BUILDDIR = os.path.join(HERE, "_build")
LIB = os.path.join(LIBDIR, "libfs2gpu.so")
INCLUDE = os.path.join(ROOT, "include")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CU_SOURCES = ["api.cu", "pm_kernels.cu", "deposit_binned.cu",
              "cola_kernels.cu", "lpt_kernels.cu",
              "noalloc.cu", "fft_pipeline.cu", "adjoint_kernels.cu",
              "api_diff.cu", "ensemble.cu"]
# files whose arithmetic need not follow the reference's rounding order may
# contract products into FMAs (the FFT butterflies)
FMAD = {"fft_pipeline.cu"}
CPP_SOURCES = ["cosmology.cpp", "power.cpp"]
HEADERS = [os.path.join(CSRC, "internal.h"), os.path.join(CSRC, "probe.h"),
           os.path.join(CSRC, "reduce_pair.cuh"),
           os.path.join(CSRC, "cola_math.cuh"),
           os.path.join(INCLUDE, "fs2gpu.h")]


def _ext_suffix() -> str:
    return sysconfig.get_config_var("EXT_SUFFIX") or ".so"


EXT = os.path.join(HERE, "fs", "_fs" + _ext_suffix())


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def build_lib(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(BUILDDIR, exist_ok=True)
    objs = []
    common = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I", INCLUDE,
              "-I", CSRC]
    for src in CU_SOURCES + CPP_SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILDDIR, src + ".o")
        objs.append(obj)
        if force or _stale(obj, [path] + HEADERS):
            if src.endswith(".cu"):
                fmad = "--fmad=true" if src in FMAD else "--fmad=false"
                cmd = [NVCC] + ARCH + common + [
                    "-lineinfo", fmad, "-Xptxas", "-v" if verbose
                    else "-O3", "-c", path, "-o", obj]
            else:
                cmd = ["g++", "-O3", "-std=c++17", "-fPIC", "-I", INCLUDE, "-I", CSRC,
                       "-I", os.path.join(CUDA_HOME, "include"), "-c", path,
                       "-o", obj]
            _run(cmd, verbose)
    if force or _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + [
            "-L", os.path.join(CUDA_HOME, "lib64"), "-lcufft",
            "-Xlinker", "-rpath=" + os.path.join(CUDA_HOME, "lib64")]
        _run(cmd, verbose)
    return LIB


def build_ext(force: bool = False, verbose: bool = False) -> str:
    import numpy as np
    src = os.path.join(CSRC, "py_fs.cpp")
    if force or _stale(EXT, [src, LIB] + HEADERS):
        py_inc = sysconfig.get_paths()["include"]
        cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-Wall",
               "-I", py_inc, "-I", np.get_include(), "-I", INCLUDE, src,
               "-o", EXT, "-L", LIBDIR, "-lfs2gpu",
               "-Wl,-rpath,$ORIGIN/../lib"]
        _run(cmd, verbose)
    return EXT


def build(force: bool = False, verbose: bool = False):
    if shutil.which(NVCC) is None and not os.path.exists(NVCC):
        raise RuntimeError("nvcc not found at %s" % NVCC)
    lib = build_lib(force, verbose)
    ext = build_ext(force, verbose)
    return lib, ext


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
