"""Writes the golden fixtures of tests/golden from the CPU oracle.

The reference ships no golden output (its tests write HDF5 files locally and
ignore them, test/.gitignore), and it cannot be built here (MPI, FFTW, GSL and
HDF5 are absent), so the fixtures come from the oracle, a restatement of the
reference's loops (oracle/).  They pin the oracle against itself over time and
give the GPU tests fixed numbers to meet.

Case `cola_16p_32m`: nc=16 particles per dimension, a 32^3 PM mesh
(pm_factor 2), box 32 Mpc/h, Omega_m = 0.31, the Eisenstein-Hu no-wiggle P(k)
of fs2_b200.power_eh, uniform draws from numpy's PCG64 with seed 7, 2LPT at
a = 0.1 ('cola'), then 3 COLA steps to a = 0.4 with the schedule of
script/cola.py.  Stored: the draws, the initial positions and dx1, the density and forces of
the first step, and x, v after the last step.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle  # noqa: E402
from fs2_b200 import power_eh  # noqa: E402

CASE = dict(nc=16, n=32, boxsize=32.0, omega_m=0.31, a_init=0.1, a_final=0.4,
            nstep=3, draw_seed=7)


def draws(nc, seed):
    rng = np.random.default_rng(seed)
    shape = (nc, nc, nc // 2)
    u_phase = rng.random(shape)
    u_ampl = 1.0 - rng.random(shape)          # in (0, 1]
    return u_phase, u_ampl


def run(case=CASE):
    nc, n, L = case["nc"], case["n"], case["boxsize"]
    k, P = power_eh.eh_nowiggle_table()
    ps = oracle.PowerSpectrum(k=k, P=P)
    cosmo = oracle.Cosmology(case["omega_m"])
    up, ua = draws(nc, case["draw_seed"])
    p = oracle.lpt(nc, L, case["a_init"], up, ua, ps, cosmo, "cola")
    x0 = p.x.copy()
    dx1 = p.dx1.copy()
    pm = oracle.PM(n, n / nc, L)
    a0, a1, ns = case["a_init"], case["a_final"], case["nstep"]
    for i in range(ns):
        a_vel = a0 + (a1 - a0) / ns * (i + 0.5)
        if i == 0:
            # fs.pm.force of the first step, with the density kept
            oracle.wrap(p.x, L)
            delta0 = oracle.unpad(pm.density(p.x)).copy()
            p.f = pm.force(p.x)
            p.a_f = p.a_x
            f0 = p.f.copy()
        else:
            oracle.pm_force(p, pm)
        oracle.cola_kick(p, cosmo, a_vel)
        a_pos = a0 + (a1 - a0) / ns * (i + 1.0)
        oracle.cola_drift(p, cosmo, a_pos)
    return dict(u_phase=up, u_ampl=ua, x0=x0, dx1=dx1, delta0=delta0, f0=f0,
                x=p.x, v=p.v)


if __name__ == "__main__":
    out = run()
    path = os.path.join(HERE, "cola_16p_32m.npz")
    np.savez_compressed(path, **out, **{"case_" + a: b for a, b in CASE.items()})
    print("wrote", path, os.path.getsize(path), "bytes")
