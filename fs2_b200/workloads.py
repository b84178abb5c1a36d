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
