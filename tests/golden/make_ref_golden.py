"""Writes tests/golden/ref_cola_16p_32m.npz from the reference's own code.

The reference ships no golden output (its tests write HDF5 files locally and
ignore them, test/.gitignore).  This script runs the reference's py/lpt.cpp,
py/pm.cpp and py/cola.cpp, compiled from its sources into oracle/_ref (see
oracle/ref.py; single-rank stand-ins for MPI, FFTW and GSL), through the
time loop of script/cola.py, and stores what they computed.  The GPU tests
and the oracle are then checked against the reference's numbers.

Case `ref_cola_16p_32m`: nc=16 particles per dimension, a 32^3 PM mesh
(pm_factor 2), box 32 Mpc/h, Omega_m = 0.31, the Eisenstein-Hu no-wiggle
P(k) of fs2_b200.power_eh written as a `k P` table, 2LPT at a = 0.1
('cola') from seed 7 of the stand-in stream, then 3 COLA steps to a = 0.4.
Stored: the draws every mode received (u_phase, u_ampl: what
fs.lpt.init_from_draws and the oracle take), the initial x, dx1, dx2, the
density and forces of the first step, and x, v after the last step.

    python tests/golden/make_ref_golden.py     (needs the reference sources)
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import ref  # noqa: E402
from fs2_b200 import power_eh  # noqa: E402

CASE = dict(nc=16, n=32, boxsize=32.0, omega_m=0.31, a_init=0.1, a_final=0.4,
            nstep=3, seed=7)


def run(case=CASE):
    if ref.lib() is None:
        raise RuntimeError("needs the reference sources or oracle/_ref")
    nc, n, L = case["nc"], case["n"], case["boxsize"]
    ref.init(case["omega_m"])
    d = tempfile.mkdtemp(prefix="fs2ref_")
    table = os.path.join(d, "pk.dat")
    power_eh.write_eh_nowiggle(table)
    a0, a1, ns = case["a_init"], case["a_final"], case["nstep"]
    x, v, d1, d2, ids, up, ua, _ = ref.lpt(nc, L, a0, case["seed"], table,
                                           "cola")
    out = dict(u_phase=up, u_ampl=ua, x0=x.copy(), dx1=d1.copy(),
               dx2=d2.copy(), id=ids)
    ref.pm_init(n, n / nc, L)
    a_x = a_v = a0
    for i in range(ns):
        a_vel = a0 + (a1 - a0) / ns * (i + 0.5)
        a_pos = a0 + (a1 - a0) / ns * (i + 1.0)
        # fs.pm.force: wrap, density, force (py/fs/pm.py:17-31)
        if i == 0:
            mesh, _ = ref.pm_density(x, n, wrap=True)
            out["delta0"] = np.ascontiguousarray(mesh[:, :, :n])
        f, _, _, x = ref.pm_force(x, n, wrap=True)
        if i == 0:
            out["f0"] = f.copy()
        v = ref.cola_kick(v, f, d1, d2, a_x, a_v, a_vel)
        a_v = a_vel
        x = ref.cola_drift(x, v, d1, d2, a_x, a_v, a_pos)
        a_x = a_pos
    out["x"], out["v"] = x, v
    return out


if __name__ == "__main__":
    res = run()
    path = os.path.join(HERE, "ref_cola_16p_32m.npz")
    np.savez_compressed(path, **res,
                        **{"case_" + a: b for a, b in CASE.items()})
    print("wrote", path, os.path.getsize(path), "bytes")
