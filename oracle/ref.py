"""The reference's own PM / COLA / 2LPT code, compiled from its sources.

TEST INFRASTRUCTURE ONLY.  tests/ use it to pin the oracle (fs2_oracle.c,
oracle.py) to the reference's arithmetic; nothing in the product imports,
links or runs it.

Recipe: g++ compiles these files of the reference tree where they lie
(default /root/reference/py, or $FS2_REFERENCE/py) --

    pm.cpp cola.cpp lpt.cpp fft.cpp cosmology.cpp power.cpp particle.cpp
    util.cpp mem.cpp msg.cpp comm.cpp config.cpp

-- together with oracle/ref_pin/stubs.cpp (single-rank MPI; FFTW 3 MPI
plans executed as double-precision DFTs; GSL quadrature, natural cubic
spline and a logged uniform stream, each written from the mathematics) and
oracle/ref_pin/harness.cpp (C entry points that follow the reference's
Python wrappers on one rank).  Flags: -std=c++11 -O2 -ffp-contract=off and
no OpenMP, i.e. the reference's serial x86-64 arithmetic.  py/pm_domain.cpp
(one-sided MPI halo exchange) is not compiled: on one rank it sends nothing,
and the harness supplies its empty-buffer accessors.

The output is oracle/_ref/libfs2ref.so (git-ignored; it travels with the
tree to machines without the reference sources).  Where neither the
sources nor a prebuilt library exist, lib() returns None and the tests that
need it skip.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
LIB_PATH = os.path.join(OUT, "libfs2ref.so")
PIN = os.path.join(HERE, "ref_pin")
REF_FILES = ["pm.cpp", "cola.cpp", "lpt.cpp", "fft.cpp", "cosmology.cpp",
             "power.cpp", "particle.cpp", "util.cpp", "mem.cpp", "msg.cpp",
             "comm.cpp", "config.cpp"]
VERSION = 1


def reference_dir() -> str:
    return os.path.join(os.environ.get("FS2_REFERENCE", "/root/reference"),
                        "py")


def build(force: bool = False) -> str | None:
    """Compiles libfs2ref.so from the reference's sources; returns its path,
    or None when the sources are not on this machine and no build exists."""
    src = reference_dir()
    have_src = all(os.path.exists(os.path.join(src, f)) for f in REF_FILES)
    if not have_src:
        return LIB_PATH if os.path.exists(LIB_PATH) else None
    deps = ([os.path.join(src, f) for f in REF_FILES] +
            [os.path.join(PIN, "stubs.cpp"), os.path.join(PIN, "harness.cpp")])
    for root, _, files in os.walk(os.path.join(PIN, "include")):
        deps += [os.path.join(root, f) for f in files]
    if (not force and os.path.exists(LIB_PATH) and
            all(os.path.getmtime(LIB_PATH) >= os.path.getmtime(d)
                for d in deps)):
        return LIB_PATH
    os.makedirs(OUT, exist_ok=True)
    cmd = (["g++", "-std=c++11", "-O2", "-ffp-contract=off", "-fno-fast-math",
            "-fPIC", "-shared", "-w",
            "-I", os.path.join(PIN, "include"), "-I", src] +
           [os.path.join(src, f) for f in REF_FILES] +
           [os.path.join(PIN, "stubs.cpp"), os.path.join(PIN, "harness.cpp"),
            "-o", LIB_PATH, "-lm"])
    subprocess.check_call(cmd)
    return LIB_PATH


_lib = None

_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_ulp = ctypes.POINTER(ctypes.c_ulong)


def lib():
    """The loaded library with argument types set, initialised for
    Omega_m = 0.31 (call init() for another value); None if unavailable."""
    global _lib
    if _lib is not None:
        return _lib
    path = build()
    if path is None:
        return None
    L = ctypes.CDLL(path)
    sz, i32, f64 = ctypes.c_size_t, ctypes.c_int, ctypes.c_double
    L.fs2ref_init.argtypes = [f64]
    for name in ("fs2ref_D_growth",):
        getattr(L, name).argtypes = [f64]
        getattr(L, name).restype = f64
    for name in ("fs2ref_D2_growth", "fs2ref_Dv_growth", "fs2ref_D2v_growth"):
        getattr(L, name).argtypes = [f64, f64]
        getattr(L, name).restype = f64
    L.fs2ref_pm_init.argtypes = [i32, f64, f64]
    L.fs2ref_pm_density.argtypes = [_f32p, sz, i32, _f32p]
    L.fs2ref_pm_force.argtypes = [_f32p, sz, i32, _f32p, _f32p, _f32p,
                                  _f32p, _f32p]
    L.fs2ref_cola_kick.argtypes = [_f32p, _f32p, _f32p, _f32p, sz, f64, f64,
                                   f64]
    L.fs2ref_cola_drift.argtypes = [_f32p, _f32p, _f32p, _f32p, sz, f64, f64,
                                    f64]
    L.fs2ref_cola_velocity.argtypes = [_f32p, _f32p, _f32p, sz, f64, _f32p]
    L.fs2ref_lpt.argtypes = [i32, f64, f64, ctypes.c_ulong, ctypes.c_char_p,
                             ctypes.c_char_p] + [_f32p] * 4 + [_u64p]
    L.fs2ref_rng_log_clear.argtypes = []
    L.fs2ref_rng_log_size.restype = sz
    L.fs2ref_rng_log_copy.argtypes = [_ulp, _f64p]
    if L.fs2ref_version() != VERSION:
        raise RuntimeError("stale oracle/_ref build")
    _lib = L
    init(0.31)
    return _lib


def _check(rc):
    if rc != 0:
        raise RuntimeError("the reference code raised an exception")


def init(omega_m: float):
    _check(lib().fs2ref_init(omega_m))


def _p32(a):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(_f32p)


def _opt32(a):
    return None if a is None else _p32(a)


def pm_init(n: int, pm_factor: float, boxsize: float):
    _check(lib().fs2ref_pm_init(n, pm_factor, boxsize))


def pm_density(x: np.ndarray, n: int, wrap: bool = True):
    """(padded density mesh, wrapped positions) from the reference's
    pm_compute_density after pm_init(n, ...)."""
    x = np.ascontiguousarray(x, dtype=np.float32).copy()
    mesh = np.zeros((n, n, 2 * (n // 2 + 1)), np.float32)
    _check(lib().fs2ref_pm_density(_p32(x), len(x), int(wrap), _p32(mesh)))
    return mesh, x


def pm_force(x: np.ndarray, n: int, wrap: bool = True, dk_inject=None,
             capture=False, mesh_inject=None):
    """pm_compute_force after the density of x.  Returns (f, fk, meshes,
    x): fk the three k-space force spectra entering the C2R ([n][n][n/2+1]
    complex64, kx-major) and meshes the three force meshes leaving it,
    when capture is set; x the positions after the wrap.  dk_inject ([n][n][n/2+1] complex64) replaces
    delta(k); mesh_inject (3 padded meshes) replaces the force meshes the
    gather reads."""
    x = np.ascontiguousarray(x, dtype=np.float32).copy()
    f = np.zeros_like(x)
    nk = n // 2 + 1
    fk = np.zeros((3, n, n, nk), np.complex64) if capture else None
    meshes = np.zeros((3, n, n, 2 * nk), np.float32) if capture else None
    dk = (None if dk_inject is None else
          np.ascontiguousarray(dk_inject, np.complex64).view(np.float32))
    mi = (None if mesh_inject is None else
          np.ascontiguousarray(mesh_inject, np.float32))
    _check(lib().fs2ref_pm_force(
        _p32(x), len(x), int(wrap), _p32(f), _opt32(dk),
        None if fk is None else _p32(fk.view(np.float32)),
        _opt32(meshes), _opt32(mi)))
    return f, fk, meshes, x


def cola_kick(v, f, dx1, dx2, a_x, a_v, a_vel):
    v = np.ascontiguousarray(v, np.float32).copy()
    c = [np.ascontiguousarray(a, np.float32) for a in (f, dx1, dx2)]
    _check(lib().fs2ref_cola_kick(_p32(v), *[_p32(a) for a in c], len(v),
                                  a_x, a_v, a_vel))
    return v


def cola_drift(x, v, dx1, dx2, a_x, a_v, a_pos):
    x = np.ascontiguousarray(x, np.float32).copy()
    c = [np.ascontiguousarray(a, np.float32) for a in (v, dx1, dx2)]
    _check(lib().fs2ref_cola_drift(_p32(x), *[_p32(a) for a in c], len(x),
                                   a_x, a_v, a_pos))
    return x


def cola_velocity(v, dx1, dx2, a_x):
    c = [np.ascontiguousarray(a, np.float32) for a in (v, dx1, dx2)]
    out = np.empty_like(c[0])
    _check(lib().fs2ref_cola_velocity(*[_p32(a) for a in c], len(out), a_x,
                                      _p32(out)))
    return out


def lpt(nc: int, boxsize: float, a: float, seed: int, pk_file: str,
        kind: str = "cola"):
    """py_lpt with the logged stand-in stream.  Returns (x, v, dx1, dx2, id,
    u_phase, u_ampl): the particles and the (nc, nc, nc/2) draws each mode
    received (the layout the oracle and fs.lpt.init_from_draws take)."""
    L = lib()
    L.fs2ref_rng_log_clear()
    np_ = nc ** 3
    x, v, d1, d2 = (np.zeros((np_, 3), np.float32) for _ in range(4))
    ids = np.zeros(np_, np.uint64)
    _check(L.fs2ref_lpt(nc, boxsize, a, seed, pk_file.encode(),
                        kind.encode(), _p32(x), _p32(v), _p32(d1), _p32(d2),
                        ids.ctypes.data_as(_u64p)))
    m = L.fs2ref_rng_log_size()
    seeds = np.zeros(m, np.uint64)
    u = np.zeros(m, np.float64)
    L.fs2ref_rng_log_copy(seeds.ctypes.data_as(_ulp), u.ctypes.data_as(_f64p))
    # the seed table takes nc^2 draws (py/lpt.cpp:241-272), then each of the
    # nc^2 columns two per iz < nc/2 (no zero amplitude was redrawn: the
    # count checks it)
    assert m == nc * nc + nc ** 3, m
    cols = u[nc * nc:].reshape(nc, nc, nc // 2, 2)
    return (x, v, d1, d2, ids, np.ascontiguousarray(cols[..., 0]),
            np.ascontiguousarray(cols[..., 1]), seeds)
