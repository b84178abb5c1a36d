"""The synthetic workloads the benchmarks and parity tests run.

All inputs are generated here from seeds: a linear P(k) table from the
Eisenstein-Hu no-wiggle fit (Omega_m=0.31, Omega_b=0.049, h=0.67, n_s=0.96,
sigma_8=0.81) written in the two-column `k P` format the reference reads, a
Gaussian random field from a seed, 2LPT particles on a grid, and the COLA
time schedule of the reference's driver script (script/cola.py:37-44).
"""
from __future__ import annotations

import os
import tempfile
from dataclasses import dataclass

OMEGA_M = 0.31


@dataclass(frozen=True)
class Workload:
    name: str
    nc: int            # particles per dimension
    n: int             # PM mesh cells per dimension
    boxsize: float     # Mpc/h
    a_init: float
    a_final: float
    nstep: int
    seed: int

    @property
    def pm_factor(self) -> float:
        return self.n / self.nc

    @property
    def np(self) -> int:
        return self.nc ** 3

    def schedule(self):
        """(a_vel, a_pos) of each step, as script/cola.py:37-44."""
        out = []
        da = (self.a_final - self.a_init) / self.nstep
        for i in range(self.nstep):
            out.append((self.a_init + da * (i + 0.5),
                        self.a_init + da * (i + 1.0)))
        return out


# plain 2LPT + COLA, 64^3 particles on 128^3, 64 Mpc/h, a = 0.1 -> 1, 10 steps
CONFIG1 = Workload("cola_64p_128m_L64", 64, 128, 64.0, 0.1, 1.0, 10, 1)
# PM force only: 256^3 on 512^3, 256 Mpc/h, 2LPT positions at a = 0.5
CONFIG2 = Workload("pm_force_256p_512m_L256", 256, 512, 256.0, 0.5, 0.5, 0, 1)
# COLA at scale: 512^3 on 1024^3, 512 Mpc/h, a = 0.02 -> 1, 10 steps
CONFIG3 = Workload("cola_512p_1024m_L512", 512, 1024, 512.0, 0.02, 1.0, 10, 1)
# differentiable: 128^3 on 256^3, 128 Mpc/h, white noise seed 2, 10 steps
CONFIG4 = Workload("adjoint_128p_256m_L128", 128, 256, 128.0, 0.1, 1.0, 10, 2)

_TABLE = None


def lpt_draws(nc: int, seed: int):
    """The uniform (phase, amplitude) draws fs.lpt.init(nc, ..., seed) uses,
    as (nc, nc, nc/2) float64 arrays, computed here with numpy: each (ix, iy)
    column has a SplitMix64 stream (Steele, Lea & Flood 2014) keyed by
    (seed, signed kx, signed ky); phase = output 2 iz + 1, amplitude =
    output 2 iz + 2, u = ((h >> 11) + 0.5) 2^-53.  Lets a caller that must
    not run the library (the CPU reference arm of the benchmark) build the
    same initial conditions."""
    import numpy as np
    M = np.uint64
    G = np.array([0x9E3779B97F4A7C15], dtype=M)

    def mix(z):
        z = (z ^ (z >> M(30))) * M(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> M(27))) * M(0x94D049BB133111EB)
        return z ^ (z >> M(31))

    with np.errstate(over="ignore"):
        i = np.arange(nc, dtype=np.int64)
        sk = np.where(i < nc // 2, i, i - nc).astype(np.uint32).astype(M)
        s = mix(np.array([seed], dtype=M) + G)
        c = (sk[:, None] << M(32)) | sk[None, :]
        col = mix(s ^ mix(c + M(0x632BE59BD9B4E019)))
        j = 2 * np.arange(nc // 2, dtype=M)

        def u(h):
            return ((h >> M(11)).astype(np.float64) + 0.5) * \
                (1.0 / 9007199254740992.0)

        up = u(mix(col[..., None] + (j + M(1)) * G))
        ua = u(mix(col[..., None] + (j + M(2)) * G))
    return up, ua


def eh_table_path(directory: str | None = None) -> str:
    """Writes (once per process) the EH no-wiggle table and returns its path."""
    global _TABLE
    if directory is None and _TABLE is not None and os.path.exists(_TABLE):
        return _TABLE
    from . import power_eh
    d = directory or tempfile.mkdtemp(prefix="fs2b200_")
    path = os.path.join(d, "eh_nowiggle_pk.dat")
    power_eh.write_eh_nowiggle(path)
    if directory is None:
        _TABLE = path
    return path
