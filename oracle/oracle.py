"""CPU oracle for the fs2 particle-mesh / COLA / 2LPT path.

TEST INFRASTRUCTURE ONLY.  Only tests/, the smoke check and the CPU-baseline
leg of bench.py import this module; the product path never does.

It restates the reference (LBJ-Wade/fs2, py/*.cpp) on the CPU:

* particle and k-space loops in C (oracle/fs2_oracle.c, built into
  oracle/_build/libfs2oracle.so), with the reference's float/double
  promotion pattern;
* 3-D FFTs with pocketfft (scipy.fft) in float32, unnormalised both ways as
  FFTW is (py/fft.cpp:80-100).  pocketfft's multi-dimensional C2R transforms
  x and y first and takes the real part along z, which is FFTW's rdft2
  behaviour on a spectrum that is not Hermitian on the kz=0 and kz=n/2 planes;
* host FP64 cosmology (py/cosmology.cpp:24-171) with scipy.integrate.quad in
  place of GSL qag, and the P(k) table (py/power.cpp:15-170) with a natural
  cubic spline from scipy in place of gsl_interp_cspline;
* FP64 answers that the float32 results' errors are reported against: the PM
  force (PM64), the COLA time loop (cola_run64) and the 2LPT chain (lpt64),
  each in float64 throughout.

Third-party arithmetic the reference takes from libraries that are not in the
reference tree: FFTW 3 (fftwf_mpi_*; any 3.3.x), GSL (gsl_integration_qag,
gsl_interp_cspline, gsl_rng_ranlxd1; any 2.x).  The GSL random stream is not
restated: the uniform draws of py/lpt.cpp:322-326 are an input here.

Parity is pinned to the reference's own known-answer tests (see the header of
fs2_oracle.c); the reference ships no golden output files.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from dataclasses import dataclass

import numpy as np
import scipy.fft as sfft
import scipy.integrate as sint
import scipy.interpolate as sinterp

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libfs2oracle.so")
ORACLE_VERSION = 4

_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)
_u64p = ctypes.POINTER(ctypes.c_uint64)


def build(force: bool = False) -> str:
    """Compile fs2_oracle.c (gcc, -ffp-contract=off, OpenMP)."""
    src = os.path.join(HERE, "fs2_oracle.c")
    if (not force and os.path.exists(LIB_PATH)
            and os.path.getmtime(LIB_PATH) >= os.path.getmtime(src)):
        return LIB_PATH
    os.makedirs(os.path.dirname(LIB_PATH), exist_ok=True)
    cmd = ["gcc", "-O2", "-std=c11", "-ffp-contract=off", "-fno-fast-math",
           "-fopenmp", "-fPIC", "-shared", src, "-o", LIB_PATH, "-lm"]
    subprocess.check_call(cmd)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB_PATH)
        if L.or_version() != ORACLE_VERSION:
            build(force=True)
            L = ctypes.CDLL(LIB_PATH)
        sz, i32, f32, f64 = (ctypes.c_size_t, ctypes.c_int, ctypes.c_float,
                             ctypes.c_double)
        L.or_periodic_wrap.argtypes = [_f32p, sz, f32]
        L.or_clear_density.argtypes = [_f32p, i32]
        L.or_cic_deposit.argtypes = [_f32p, sz, _f32p, i32, f32, f64, i32]
        L.or_force_gather.argtypes = [_f32p, sz, _f32p, i32, f32, i32, _f32p,
                                      i32]
        L.or_force_mesh_k.argtypes = [_f32p, _f32p, i32, f32, i32, i32]
        L.or_cola_kick.argtypes = [_f32p, _f32p, _f32p, _f32p, sz, f64, f32,
                                   f32, f32, i32]
        L.or_cola_drift.argtypes = [_f32p, _f32p, _f32p, _f32p, sz, f64, f32,
                                    f32, i32]
        L.or_leapfrog_velocity.argtypes = [_f32p, _f32p, _f32p, sz, f32, f32]
        L.or_leapfrog_kick.argtypes = [_f32p, _f32p, sz, f64, f32]
        L.or_leapfrog_drift.argtypes = [_f32p, _f32p, sz, f64]
        L.or_lpt_psi_k.argtypes = [i32, f64, _f64p, _f64p, _f64p, _f64p, i32,
                                   _f32p, _f32p, _f32p]
        L.or_lpt_psi_ij_k.argtypes = [i32, f64] + [_f32p] * 9
        L.or_lpt_source.argtypes = [i32] + [_f32p] * 7
        L.or_lpt_psi2_k.argtypes = [i32, f64, _f32p, _f32p, _f32p, _f32p]
        L.or_lpt_set_particles.argtypes = (
            [i32, f64, f32] + [_f32p] * 6 + [f32] * 4 + [_f32p] * 4 + [_u64p])
        L.or_cola_velocity.argtypes = [_f32p, _f32p, _f32p, sz, f32, f32,
                                       _f32p]
        L.or_cic_deposit_f64.argtypes = [_f64p, sz, _f64p, i32, f64, f64]
        L.or_force_gather_f64.argtypes = [_f64p, sz, _f64p, i32, f64, i32,
                                          _f64p, i32]
        _lib = L
    return _lib


def _p32(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(_f32p)


def _p64(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_f64p)


def n_threads_default() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:  # pragma: no cover
        return os.cpu_count() or 1


# --------------------------------------------------------------------------
# FFT on padded meshes (py/fft.cpp:80-100, unnormalised)
# --------------------------------------------------------------------------
def ncz_of(n: int) -> int:
    return 2 * (n // 2 + 1)


def new_mesh(n: int) -> np.ndarray:
    return np.zeros((n, n, ncz_of(n)), dtype=np.float32)


def r2c(mesh: np.ndarray, workers: int = 1) -> np.ndarray:
    """Padded real mesh -> complex64 [n][n][n/2+1] (forward, unscaled)."""
    n = mesh.shape[0]
    out = sfft.rfftn(mesh[:, :, :n], workers=workers)
    assert out.dtype == np.complex64
    return np.ascontiguousarray(out)


def c2r(fk: np.ndarray, workers: int = 1) -> np.ndarray:
    """complex64 [n][n][n/2+1] -> padded real mesh (inverse, unscaled)."""
    n = fk.shape[0]
    r = sfft.irfftn(fk, s=(n, n, n), axes=(0, 1, 2), norm="forward",
                    workers=workers)
    assert r.dtype == np.float32
    mesh = new_mesh(n)
    mesh[:, :, :n] = r
    return mesh


def cview(a: np.ndarray) -> np.ndarray:
    """complex64 array as its interleaved float32 view (for the C loops)."""
    return np.ascontiguousarray(a).view(np.float32)


# --------------------------------------------------------------------------
# Cosmology, py/cosmology.cpp:24-171 (flat LCDM, FP64)
# --------------------------------------------------------------------------
class Cosmology:
    def __init__(self, omega_m: float):
        self.om = float(omega_m)
        self._norm = 1.0 / self._growth_unnormalised(1.0)   # :222

    def hubble(self, a: float) -> float:                    # :106-110
        om = self.om
        return math.sqrt(om / (a * a * a) + (1 - om))

    def omega(self, a: float) -> float:                     # :112-117
        om = self.om
        return om / (om + (1 - om) * (a * a * a))

    def _growth_unnormalised(self, a: float) -> float:      # :153-171
        om = self.om

        def integrand(x):
            aHinv = 1.0 / math.sqrt(om / x + (1 - om) * (x * x))
            return aHinv * aHinv * aHinv

        r, _ = sint.quad(integrand, 0.0, a, epsabs=0.0, epsrel=1e-13,
                         limit=500)
        return self.hubble(a) * r

    def D(self, a: float) -> float:                         # :33-40
        if a == 0.0:
            return 0.0
        return self._norm * self._growth_unnormalised(a)

    def D2(self, a: float, D: float) -> float:              # :42-48
        if a == 0.0:
            return 0.0
        return -3.0 / 7.0 * D * D * math.pow(self.omega(a), -1.0 / 143.0)

    def f(self, a: float) -> float:                         # :73-84
        if a == 0.0:
            return 1.0
        d_un = self._growth_unnormalised(a)
        hf = self.hubble(a)
        return 1.0 / (d_un * a * a * hf * hf) - 1.5 * self.om / (hf * hf * a * a * a)

    def Dv(self, a: float, D: float) -> float:              # :50-58
        if a == 0.0:
            return 1.0
        return a * a * D * self.hubble(a) * self.f(a)

    def D2v(self, a: float, D2: float) -> float:            # :60-66
        return 2.0 * a * a * D2 * self.hubble(a) * self.f(a)

    @staticmethod
    def D2a(D1: float, D2: float) -> float:                 # :68-71
        return D2 - D1 * D1


# --------------------------------------------------------------------------
# Power spectrum table, py/power.cpp:15-170
# --------------------------------------------------------------------------
class PowerSpectrum:
    def __init__(self, filename: str | None = None, k=None, P=None):
        if filename is not None:
            k, P = read_power_file(filename)
        self.log_k = np.log(np.asarray(k, dtype=np.float64))
        self.log_P = np.log(np.asarray(P, dtype=np.float64))
        self.n = len(self.log_k)
        self._spl = sinterp.CubicSpline(self.log_k, self.log_P,
                                        bc_type="natural")

    def P(self, k):
        return np.exp(self._spl(np.log(k)))

    def spline_arrays(self):
        """Knots and the 4 x (n-1) coefficient table for the C oracle."""
        return (np.ascontiguousarray(self._spl.x, dtype=np.float64),
                np.ascontiguousarray(self._spl.c, dtype=np.float64))

    def compute_sigma(self, R: float) -> float:             # :146-170
        fac = 1.0 / (2.0 * math.pi * math.pi)
        k0 = math.exp(self.log_k[0])
        f0 = 0.0
        sigma2 = 0.0
        for i in range(self.n):
            k = math.exp(self.log_k[i])
            x = k * R
            w = 3.0 * (math.sin(x) - x * math.cos(x)) / (x * x * x)
            f1 = math.exp(self.log_P[i]) * k * k * w * w
            sigma2 += 0.5 * (f0 + f1) * (k - k0)
            k0 = k
            f0 = f1
        return math.sqrt(fac * sigma2)


def read_power_file(filename: str):
    """Reads `k P` lines the way PowerSpectrum::read_file_ does
    (py/power.cpp:57-144): '#' lines skipped, k <= 0 skipped, unsorted k is
    an error, the first unparsable line ends the table."""
    ks, Ps = [], []
    k_prev = 0.0
    with open(filename) as fp:
        for line in fp:
            if line.startswith("#"):
                continue
            parts = line.split()
            try:
                k, P = float(parts[0]), float(parts[1])
            except (IndexError, ValueError):
                break
            if k <= 0.0:
                continue
            if k < k_prev:
                raise IOError("k must be sorted in increasing order")
            ks.append(k)
            Ps.append(P)
            k_prev = k
    return np.array(ks), np.array(Ps)


# --------------------------------------------------------------------------
# Particle-mesh: py/pm.cpp
# --------------------------------------------------------------------------
class PM:
    """Module state of py/pm.cpp:22-30 for one rank."""

    def __init__(self, nc_pm: int, pm_factor: float, boxsize: float,
                 nthreads: int = 1):
        if nc_pm <= 1:
            raise RuntimeError("nc_pm must be larger than 1")   # :245-249
        if boxsize <= 0:
            raise RuntimeError("boxsize must be positive")      # :251-255
        self.n = int(nc_pm)
        self.pm_factor = float(pm_factor)
        self.boxsize = np.float32(boxsize)                      # Float
        self.nthreads = nthreads
        self.mesh = new_mesh(self.n)
        self.delta_k = None
        self.force_meshes = [None, None, None]

    def density(self, x: np.ndarray) -> np.ndarray:
        """clear_density + pm_assign_cic_density (py/pm.cpp:341-355).
        Returns the padded mesh (delta)."""
        L = lib()
        x = np.ascontiguousarray(x, dtype=np.float32)
        L.or_clear_density(_p32(self.mesh), self.n)
        L.or_cic_deposit(_p32(x), x.shape[0], _p32(self.mesh), self.n,
                         self.boxsize, self.pm_factor, self.nthreads)
        return self.mesh

    def force(self, x: np.ndarray) -> np.ndarray:
        """pm_compute_force (py/pm.cpp:306-338) after density(x).
        Returns f [np][3] float32."""
        L = lib()
        x = np.ascontiguousarray(x, dtype=np.float32)
        np_ = x.shape[0]
        f = np.zeros((np_, 3), dtype=np.float32)
        self.delta_k = r2c(self.mesh, workers=self.nthreads)     # :431-458
        dk = cview(self.delta_k)
        for axis in range(3):
            fk = np.empty_like(self.delta_k)
            L.or_force_mesh_k(_p32(dk), _p32(cview(fk)), self.n,
                              self.boxsize, axis, self.nthreads)
            fk = fk  # filled through its float view
            fmesh = c2r(fk, workers=self.nthreads)               # :507
            self.force_meshes[axis] = fmesh
            L.or_force_gather(_p32(x), np_, _p32(fmesh), self.n, self.boxsize,
                              axis, _p32(f), self.nthreads)
        # the reference's FFT buffer holds the last C2R output (f_z mesh)
        self.mesh = self.force_meshes[2].copy()
        return f


def wrap(x: np.ndarray, boxsize) -> np.ndarray:
    """periodic_wrapup_p over all particles (py/util.h:14-24), in place."""
    x32 = np.ascontiguousarray(x, dtype=np.float32)
    lib().or_periodic_wrap(_p32(x32), x32.shape[0], np.float32(boxsize))
    return x32


class PM64:
    """The PM force of py/pm.cpp:57-220,431-508 evaluated in float64 from
    float64 positions: deposit, R2C, the k-space gradient (same wavenumber
    and Nyquist conventions), C2R and gather.  Not the reference's float
    arithmetic: the answer the float32 paths' errors are reported against."""

    def __init__(self, nc_pm: int, pm_factor: float, boxsize: float,
                 nthreads: int = 1):
        self.n = int(nc_pm)
        self.pm_factor = float(pm_factor)
        self.boxsize = float(boxsize)
        self.nthreads = nthreads
        self.mesh = np.zeros((self.n, self.n, ncz_of(self.n)), np.float64)
        self.force_meshes = [None, None, None]

    def density(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64)
        lib().or_cic_deposit_f64(_p64(x), x.shape[0], _p64(self.mesh),
                                 self.n, self.boxsize, self.pm_factor)
        return self.mesh

    def force(self, x: np.ndarray) -> np.ndarray:
        n = self.n
        x = np.ascontiguousarray(x, dtype=np.float64)
        f = np.zeros((x.shape[0], 3), np.float64)
        dk = sfft.rfftn(self.mesh[:, :, :n], workers=self.nthreads)
        i = np.arange(n)
        kxy = np.where(i <= n // 2, i, i - n).astype(np.float64)   # :483,489
        kz = np.arange(n // 2 + 1, dtype=np.float64)
        K = (kxy[:, None, None], kxy[None, :, None], kz[None, None, :])
        k2 = K[0] ** 2 + K[1] ** 2 + K[2] ** 2
        k2[0, 0, 0] = 1.0
        f1 = -1.0 / float(n) ** 3 / (2.0 * math.pi / self.boxsize)
        for axis in range(3):
            fk = (1j * (f1 / k2 * K[axis])) * dk
            fk[0, 0, 0] = 0.0
            r = sfft.irfftn(fk, s=(n, n, n), axes=(0, 1, 2), norm="forward",
                            workers=self.nthreads)
            mesh = np.zeros((n, n, ncz_of(n)), np.float64)
            mesh[:, :, :n] = r
            self.force_meshes[axis] = mesh
            lib().or_force_gather_f64(_p64(x), x.shape[0], _p64(mesh), n,
                                      self.boxsize, axis, _p64(f),
                                      self.nthreads)
        return f


def unpad(mesh: np.ndarray) -> np.ndarray:
    n = mesh.shape[0]
    return np.ascontiguousarray(mesh[:, :, :n])


# --------------------------------------------------------------------------
# COLA: py/cola.cpp
# --------------------------------------------------------------------------
N_LPT = -2.5   # py/cola.cpp:20 (a float literal, exactly -2.5)


def kick_coefficients(cosmo: Cosmology, a_v: float, a_x: float,
                      a_vel: float):
    """Host part of cola_kick, py/cola.cpp:50-66."""
    ai, a, af = a_v, a_x, a_vel
    om = cosmo.om
    kick_factor = np.float32((af ** N_LPT - ai ** N_LPT) /
                             (N_LPT * a ** N_LPT *
                              math.sqrt(om / a + (1.0 - om) * a * a)))
    g1 = cosmo.D(a)
    g2 = cosmo.D2(a, g1)
    q1 = np.float32(g1)
    q2 = np.float32(Cosmology.D2a(g1, g2))
    return om, kick_factor, q1, q2


def Sq(cosmo: Cosmology, ai: float, af: float, av: float) -> float:
    """py/cola.cpp:152-179: int_ai^af a^n/(a^3 H) da / av^n."""
    om = cosmo.om

    def fun(a):
        return a ** N_LPT / (math.sqrt(om / (a * a * a) + 1.0 - om) * a * a * a)

    r, _ = sint.quad(fun, ai, af, epsabs=0.0, epsrel=1e-13, limit=500)
    return r / av ** N_LPT


def drift_coefficients(cosmo: Cosmology, a_x: float, a_v: float,
                       a_pos: float):
    """Host part of cola_drift, py/cola.cpp:96-109."""
    ai, af = a_x, a_pos
    dt = Sq(cosmo, ai, af, a_v)
    gi = cosmo.D(ai)
    gf = cosmo.D(af)
    da1 = np.float32(gf - gi)
    da2 = np.float32(cosmo.D2(af, gf) - cosmo.D2(ai, gi))
    return dt, da1, da2


@dataclass
class ParticleState:
    x: np.ndarray
    v: np.ndarray
    dx1: np.ndarray
    dx2: np.ndarray
    id: np.ndarray
    a_x: float
    a_v: float
    a_f: float = 0.0
    boxsize: float = 0.0
    f: np.ndarray | None = None

    def copy(self):
        return ParticleState(self.x.copy(), self.v.copy(), self.dx1.copy(),
                             self.dx2.copy(), self.id.copy(), self.a_x,
                             self.a_v, self.a_f, self.boxsize,
                             None if self.f is None else self.f.copy())


def cola_kick(p: ParticleState, cosmo: Cosmology, a_vel: float,
              nthreads: int = 1):
    om, kf, q1, q2 = kick_coefficients(cosmo, p.a_v, p.a_x, a_vel)
    lib().or_cola_kick(_p32(p.f), _p32(p.dx1), _p32(p.dx2), _p32(p.v),
                       p.x.shape[0], om, kf, q1, q2, nthreads)
    p.a_v = a_vel


def cola_drift(p: ParticleState, cosmo: Cosmology, a_pos: float,
               nthreads: int = 1):
    dt, da1, da2 = drift_coefficients(cosmo, p.a_x, p.a_v, a_pos)
    lib().or_cola_drift(_p32(p.x), _p32(p.v), _p32(p.dx1), _p32(p.dx2),
                        p.x.shape[0], dt, da1, da2, nthreads)
    p.a_x = a_pos


def cola_velocity(p: ParticleState, cosmo: Cosmology, Dv=None,
                  D2v=None) -> np.ndarray:
    """cola_velocity, py/cola.cpp:129-148: the COLA velocity with the 2LPT
    part restored.  D1 is passed where D2 is expected (:138), as the
    reference does.  Dv and D2v (Float) may be given to run the loop with
    another implementation's coefficients."""
    a = p.a_x
    D1 = cosmo.D(a)
    Dv = np.float32(cosmo.Dv(a, D1) if Dv is None else Dv)
    D2v = np.float32(cosmo.D2v(a, D1) if D2v is None else D2v)
    out = np.empty_like(p.v)
    lib().or_cola_velocity(_p32(p.v), _p32(p.dx1), _p32(p.dx2),
                           p.v.shape[0], Dv, D2v, _p32(out))
    return out


# --------------------------------------------------------------------------
# Leapfrog (non-COLA): py/leapfrog.cpp
# --------------------------------------------------------------------------
def leapfrog_Sphi(cosmo: Cosmology, ai: float, af: float) -> float:
    """py/leapfrog.cpp:97-121: int_ai^af da / (a^2 H(a))."""
    om = cosmo.om
    r, _ = sint.quad(lambda a: 1.0 / (math.sqrt(om / a ** 3 + 1.0 - om) * a * a),
                     ai, af, epsabs=0.0, epsrel=1e-13, limit=500)
    return r


def leapfrog_Sq(cosmo: Cosmology, ai: float, af: float) -> float:
    """py/leapfrog.cpp:123-146: int_ai^af da / (a^3 H(a))."""
    om = cosmo.om
    r, _ = sint.quad(lambda a: 1.0 / (math.sqrt(om / a ** 3 + 1.0 - om) * a ** 3),
                     ai, af, epsabs=0.0, epsrel=1e-13, limit=500)
    return r


def leapfrog_initial_velocity(p: ParticleState, cosmo: Cosmology, a: float):
    """leapfrog_set_initial_velocity, py/leapfrog.cpp:18-39."""
    da1 = np.float32(cosmo.D(a))
    da2 = np.float32(cosmo.D2(a, float(da1)))
    dv = np.float32(cosmo.Dv(a, float(da1)))
    d2v = np.float32(cosmo.D2v(a, float(da2)))
    lib().or_leapfrog_velocity(_p32(p.dx1), _p32(p.dx2), _p32(p.v),
                               p.x.shape[0], dv, d2v)
    p.a_v = a


def leapfrog_kick(p: ParticleState, cosmo: Cosmology, a_vel: float):
    """leapfrog_kick, py/leapfrog.cpp:41-68."""
    kf = np.float32(leapfrog_Sphi(cosmo, p.a_v, a_vel))
    lib().or_leapfrog_kick(_p32(p.f), _p32(p.v), p.x.shape[0], cosmo.om, kf)
    p.a_v = a_vel


def leapfrog_drift(p: ParticleState, cosmo: Cosmology, a_pos: float):
    """leapfrog_drift, py/leapfrog.cpp:70-95."""
    dt = leapfrog_Sq(cosmo, p.a_x, a_pos)
    lib().or_leapfrog_drift(_p32(p.x), _p32(p.v), p.x.shape[0], dt)
    p.a_x = a_pos


def pm_force(p: ParticleState, pm: PM):
    """fs.pm.force (py/fs/pm.py:17-31): wrap, density, force, with the
    a_f == a_x cache of py/pm.cpp:311."""
    lib().or_periodic_wrap(_p32(p.x), p.x.shape[0], pm.boxsize)
    pm.density(p.x)
    if p.a_f == p.a_x and p.f is not None:
        return
    p.f = pm.force(p.x)
    p.a_f = p.a_x


def cola_run(p: ParticleState, pm: PM, cosmo: Cosmology, a_init: float,
             a_final: float, nstep: int, nthreads: int = 1):
    """The time loop of script/cola.py:37-44."""
    for i in range(nstep):
        a_vel = a_init + (a_final - a_init) / nstep * (i + 0.5)
        pm_force(p, pm)
        cola_kick(p, cosmo, a_vel, nthreads)
        a_pos = a_init + (a_final - a_init) / nstep * (i + 1.0)
        cola_drift(p, cosmo, a_pos, nthreads)
    return p


def cola_run64(p: ParticleState, pm64: PM64, cosmo: Cosmology,
               schedule) -> ParticleState:
    """The same time loop (script/cola.py:37-44) entirely in float64: the
    state in float64, the wrap of py/util.h:14-24, PM64's force, and the
    kick and drift of py/cola.cpp:48-127 with their coefficients kept in
    double (no Float rounding anywhere).  Not the reference's arithmetic:
    the answer a float32 run's final positions and velocities are reported
    against.  `schedule` is the (a_vel, a_pos) list; returns a new state."""
    L = pm64.boxsize
    x = np.asarray(p.x, np.float64).copy()
    v = np.asarray(p.v, np.float64).copy()
    d1 = np.asarray(p.dx1, np.float64)
    d2 = np.asarray(p.dx2, np.float64)
    a_x, a_v = p.a_x, p.a_v
    om = cosmo.om
    for a_vel, a_pos in schedule:
        x = np.where(x < 0, x + L, np.where(x >= L, x - L, x))
        pm64.density(x)
        f = pm64.force(x)
        # kick, py/cola.cpp:50-66,80-86
        kf = ((a_vel ** N_LPT - a_v ** N_LPT) /
              (N_LPT * a_x ** N_LPT *
               math.sqrt(om / a_x + (1.0 - om) * a_x * a_x)))
        g1 = cosmo.D(a_x)
        q2 = Cosmology.D2a(g1, cosmo.D2(a_x, g1))
        v = v + kf * (-1.5 * om) * (f + g1 * d1 + q2 * d2)
        a_v = a_vel
        # drift, py/cola.cpp:96-123
        dt = Sq(cosmo, a_x, a_pos, a_v)
        gi, gf = cosmo.D(a_x), cosmo.D(a_pos)
        da1 = gf - gi
        da2 = cosmo.D2(a_pos, gf) - cosmo.D2(a_x, gi)
        x = x + v * dt + (d1 * da1 + d2 * da2)
        a_x = a_pos
    return ParticleState(x, v, d1.copy(), d2.copy(), p.id.copy(), a_x=a_x,
                         a_v=a_v, a_f=0.0, boxsize=L)


# --------------------------------------------------------------------------
# 2LPT: py/lpt.cpp
# --------------------------------------------------------------------------
def seedtable(nc: int, u: np.ndarray) -> np.ndarray:
    """set_seedtable, py/lpt.cpp:235-273 (from N-GenIC): the nc*nc column
    seeds, filled from the uniform draws u (in the order drawn) as
    (unsigned int)(0x7fffffff*u), in the reference's symmetric order."""
    t = np.zeros(nc * nc, np.uint32)
    it = iter(u)

    def put(idx):
        t[idx] = np.uint32(int(0x7fffffff * float(next(it))))

    for i in range(nc // 2):
        for j in range(i):
            put(i * nc + j)
        for j in range(i + 1):
            put(j * nc + i)
        for j in range(i):
            put((nc - 1 - i) * nc + j)
        for j in range(i + 1):
            put((nc - 1 - j) * nc + i)
        for j in range(i):
            put(i * nc + (nc - 1 - j))
        for j in range(i + 1):
            put(j * nc + (nc - 1 - i))
        for j in range(i):
            put((nc - 1 - i) * nc + (nc - 1 - j))
        for j in range(i + 1):
            put((nc - 1 - j) * nc + (nc - 1 - i))
    return t


def lpt_psi_k(nc: int, boxsize: float, u_phase: np.ndarray,
              u_ampl: np.ndarray, ps: PowerSpectrum):
    """lpt_generate_psi_k with the uniform draws given."""
    knots, coef = ps.spline_arrays()
    kz = nc // 2 + 1
    psi = [np.zeros((nc, nc, kz), dtype=np.complex64) for _ in range(3)]
    up = np.ascontiguousarray(u_phase, dtype=np.float64)
    ua = np.ascontiguousarray(u_ampl, dtype=np.float64)
    assert up.size == nc * nc * (nc // 2) and ua.size == up.size
    lib().or_lpt_psi_k(nc, float(boxsize), _p64(up), _p64(ua), _p64(knots),
                       _p64(coef), len(knots), *[_p32(cview(a)) for a in psi])
    return psi


def psi_from_delta_k(nc: int, boxsize: float, delta_k: np.ndarray):
    """psi_i(k) = i k_i/k^2 delta(k) with the LPT wavenumbers
    (py/lpt.cpp:333-346, :374-375), zero on the Nyquist planes and at k=0 as
    lpt_generate_psi_k leaves them (:328-331).  Used for a delta(k) that is
    given directly (e.g. from white noise)."""
    dk = 2.0 * math.pi / boxsize
    i = np.arange(nc)
    kx = np.where(i < nc // 2, dk * i, -dk * (nc - i))
    kzv = kx[: nc // 2 + 1]
    K = np.meshgrid(kx, kx, kzv, indexing="ij")
    k2 = K[0] ** 2 + K[1] ** 2 + K[2] ** 2
    k2[0, 0, 0] = 1.0
    d = delta_k.astype(np.complex128)
    out = []
    for a in range(3):
        p = 1j * K[a] / k2 * d
        p[nc // 2, :, :] = 0
        p[:, nc // 2, :] = 0
        p[:, :, nc // 2] = 0
        p[0, 0, 0] = 0
        out.append(p.astype(np.complex64))
    return out


def lpt_from_psi_k(nc: int, boxsize: float, a: float, psi_k, cosmo: Cosmology,
                   kind: str = "cola", offset: float = 0.5,
                   workers: int = 1) -> ParticleState:
    """lpt_compute_psi2_k + lpt_set_displacements (py/lpt.cpp:100-225,
    439-591) from psi(k)."""
    L = lib()
    psi_k = [np.ascontiguousarray(p, dtype=np.complex64) for p in psi_k]
    kz = nc // 2 + 1
    ij = [np.empty((nc, nc, kz), dtype=np.complex64) for _ in range(6)]
    L.or_lpt_psi_ij_k(nc, float(boxsize), *[_p32(cview(p)) for p in psi_k],
                      *[_p32(cview(q)) for q in ij])
    ij_x = [c2r(q, workers) for q in ij]                          # :515-516
    div = new_mesh(nc)
    L.or_lpt_source(nc, *[_p32(m) for m in ij_x], _p32(div))        # :522-535
    div_k = r2c(div, workers)                                      # :542
    psi2_k = [np.empty((nc, nc, kz), dtype=np.complex64) for _ in range(3)]
    L.or_lpt_psi2_k(nc, float(boxsize), _p32(cview(div_k)),
                    *[_p32(cview(q)) for q in psi2_k])
    psi_x = [c2r(p, workers) for p in psi_k]                       # :132-135
    psi2_x = [c2r(q, workers) for q in psi2_k]

    D1 = np.float32(cosmo.D(a))                                    # :156-173
    D2 = np.float32(0.0 if kind == "zeldovich" else cosmo.D2(a, float(D1)))
    if kind == "cola":
        Dv = D2v = np.float32(0.0)
    elif kind == "zeldovich":
        Dv = np.float32(cosmo.Dv(a, float(D1)))
        D2v = np.float32(0.0)
    elif kind == "2lpt":
        Dv = np.float32(cosmo.Dv(a, float(D1)))
        D2v = np.float32(cosmo.D2v(a, float(D1)))   # D1 passed for D2 (:172)
    else:
        raise AssertionError("unknown kind %r" % kind)

    np_ = nc ** 3
    x = np.empty((np_, 3), dtype=np.float32)
    v = np.empty_like(x)
    dx1 = np.empty_like(x)
    dx2 = np.empty_like(x)
    ids = np.empty(np_, dtype=np.uint64)
    L.or_lpt_set_particles(nc, float(boxsize), np.float32(offset),
                           *[_p32(m) for m in psi_x],
                           *[_p32(m) for m in psi2_x],
                           D1, D2, Dv, D2v, _p32(x), _p32(v), _p32(dx1),
                           _p32(dx2), ids.ctypes.data_as(_u64p))
    return ParticleState(x, v, dx1, dx2, ids, a_x=a, a_v=a, a_f=0.0,
                         boxsize=boxsize)


def lpt(nc: int, boxsize: float, a: float, u_phase, u_ampl,
        ps: PowerSpectrum, cosmo: Cosmology, kind: str = "cola",
        offset: float = 0.5, workers: int = 1) -> ParticleState:
    psi_k = lpt_psi_k(nc, boxsize, u_phase, u_ampl, ps)
    return lpt_from_psi_k(nc, boxsize, a, psi_k, cosmo, kind, offset,
                          workers)


def lpt64(nc: int, boxsize: float, a: float, u_phase, u_ampl,
          ps: PowerSpectrum, cosmo: Cosmology, offset: float = 0.5):
    """The 2LPT chain of py/lpt.cpp:100-225,276-591 in float64 throughout
    (psi(k), the six derivatives, the real-space source, psi2(k), the
    inverse transforms in complex128, D1 and D2 unrounded), vectorised with
    numpy.  Not the reference's arithmetic: the answer the float32 dx1, dx2
    and x are reported against.  Returns (x, dx1, dx2) as [nc^3][3] float64
    in the particle order of lpt_set_displacements."""
    n = int(nc)
    L = float(boxsize)
    dk = 2.0 * math.pi / L
    i = np.arange(n)
    kl = np.where(i < n // 2, dk * i, -dk * (n - i))     # LPT convention
    up = np.asarray(u_phase, np.float64).reshape(n, n, n // 2)
    ua = np.asarray(u_ampl, np.float64).reshape(n, n, n // 2)

    # psi(k), py/lpt.cpp:321-426
    KX, KY, KZ = np.meshgrid(kl, kl, kl[: n // 2], indexing="ij")
    k2 = KX ** 2 + KY ** 2 + KZ ** 2
    k2s = np.where(k2 > 0, k2, 1.0)
    kmag = np.sqrt(k2s)
    fac = (2 * math.pi / L) ** 1.5
    dmag = fac * np.sqrt(-np.log(ua) / (8 * math.pi ** 3) * ps.P(kmag))
    ph = 2 * math.pi * up
    base = dmag * (-np.sin(ph) + 1j * np.cos(ph)) / k2s   # times k_i
    IX, IY, IZ = np.meshgrid(i, i, i[: n // 2], indexing="ij")
    keep = ((IX != n // 2) & (IY != n // 2) &
            ~((IX == 0) & (IY == 0) & (IZ == 0)))
    psi_k = [np.zeros((n, n, n // 2 + 1), np.complex128) for _ in range(3)]
    for c, K in enumerate((KX, KY, KZ)):
        val = np.where(keep, base * K, 0.0)
        p = psi_k[c]
        p[:, :, 1: n // 2] = val[:, :, 1:]                   # iz > 0
        # kz = 0: (0, iy < n/2) and its mirror (0, n - iy); (ix < n/2, iy)
        # and its mirror (n - ix, n - iy)
        for ix in range(n // 2):
            for iy in range(n):
                if not keep[ix, iy, 0] or (ix == 0 and iy >= n // 2):
                    continue
                p[ix, iy, 0] = val[ix, iy, 0]
                p[(n - ix) % n, (n - iy) % n, 0] = np.conj(val[ix, iy, 0])

    def c2r(fk):
        return sfft.irfftn(fk, s=(n, n, n), axes=(0, 1, 2), norm="forward")

    # psi_ij(k) = i k_j psi_i(k), the source, psi2(k), py/lpt.cpp:465-586
    kz = kl[: n // 2 + 1]
    K3 = (kl[:, None, None], kl[None, :, None], kz[None, None, :])
    pairs = ((0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2))
    ij = [c2r(1j * K3[j] * psi_k[c]) for c, j in pairs]
    S = (ij[0] * (ij[3] + ij[5]) + ij[3] * ij[5]
         - ij[1] ** 2 - ij[2] ** 2 - ij[4] ** 2)
    Sk = sfft.rfftn(S)
    kk = K3[0] ** 2 + K3[1] ** 2 + K3[2] ** 2
    kk[0, 0, 0] = 1.0
    psi2 = []
    for c in range(3):
        q = -1j * K3[c] / kk * Sk
        q[0, 0, 0] = 0.0
        psi2.append(c2r(q))
    psi = [c2r(p) for p in psi_k]

    # particles, py/lpt.cpp:137-211
    D1 = cosmo.D(a)
    D2 = cosmo.D2(a, D1)
    dx1 = np.stack([p.reshape(-1) for p in psi], -1)
    dx2 = np.stack([p.reshape(-1) for p in psi2], -1) / float(n) ** 3
    g = (np.stack(np.meshgrid(i, i, i, indexing="ij"), -1).reshape(-1, 3)
         + offset) * (L / n)
    return g + D1 * dx1 + D2 * dx2, dx1, dx2
