"""The CUDA path against the reference's own code: the committed fixture
that the reference computed (tests/golden/ref_cola_16p_32m.npz, written by
tests/golden/make_ref_golden.py from the reference's sources compiled into
oracle/_ref), and, where oracle/_ref/libfs2ref.so is present, the compiled
reference itself on the same inputs.

Tolerances: density rel-L2 <= 1e-5 (and the reference's own 500 eps on the
cell values, test/test_pm_density.py:41), force rel-L2 <= 1e-4, positions
after the steps <= 1e-3 cell RMS; kick and drift bit for bit.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
OMEGA_M = 0.31


@pytest.fixture(scope="module")
def fs():
    import fs2_b200.fs as fs
    fs.cosmology.init(OMEGA_M)
    return fs


@pytest.fixture(scope="module")
def ref():
    import ref as R
    if R.lib() is None:
        pytest.skip("oracle/_ref (the compiled reference) is not available")
    R.init(OMEGA_M)
    return R


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _particles(fs, L, **fields):
    n = len(fields["x"])
    p = fs.Particles(n, L)
    for k, v in fields.items():
        p.set(k, np.ascontiguousarray(v, np.float32))
    return p


def test_reference_fixture(fs, eh_table):
    # 2LPT from the draws the reference's run received, then the time loop
    # of script/cola.py through fs.pm.force / kick / drift
    g = np.load(os.path.join(HERE, "golden", "ref_cola_16p_32m.npz"))
    nc, n, L = int(g["case_nc"]), int(g["case_n"]), float(g["case_boxsize"])
    a0, a1, ns = (float(g["case_a_init"]), float(g["case_a_final"]),
                  int(g["case_nstep"]))
    ps = fs.PowerSpectrum(eh_table)
    p = fs.lpt.init_from_draws(nc, L, a0, ps, g["u_phase"], g["u_ampl"],
                               "cola")
    assert np.array_equal(p.id, g["id"])
    assert rel_l2(p.dx1, g["dx1"]) <= 1e-5 and rel_l2(p.dx2, g["dx2"]) <= 1e-4
    fs.pm.init(n, n / nc, L)
    for i in range(ns):
        a_vel = a0 + (a1 - a0) / ns * (i + 0.5)
        fs.pm.send_positions(p)
        d = fs.pm.compute_density(p).asarray().copy()
        fs.pm.compute_force(p)
        if i == 0:
            assert rel_l2(d, g["delta0"]) <= 1e-5
            assert rel_l2(p.force, g["f0"]) <= 1e-4
        fs.cola.kick(p, a_vel)
        fs.cola.drift(p, a0 + (a1 - a0) / ns * (i + 1.0))
    dx = p.x.astype(np.float64) - g["x"]
    dx -= L * np.round(dx / L)
    rms = float(np.sqrt(np.mean(dx ** 2))) / (L / n)
    print("\nreference fixture: final x rms %.2e cell, v rel-L2 %.2e"
          % (rms, rel_l2(p.v, g["v"])))
    assert rms <= 1e-3
    assert rel_l2(p.v, g["v"]) <= 1e-4


@pytest.mark.parametrize("mode", ["atomic", "deterministic"])
def test_density_against_reference(fs, ref, mode):
    rng = np.random.default_rng(12)
    n, L = 64, 64.0
    g = (np.stack(np.meshgrid(*[np.arange(32)] * 3, indexing="ij"), -1)
         .reshape(-1, 3) + 0.5) * (L / 32)
    x = np.mod(g + rng.normal(0, 1.5, g.shape), L).astype(np.float32)
    x[:4096] = rng.normal(0.3 * L, 0.5, (4096, 3)).astype(np.float32)
    ref.pm_init(n, 2.0, L)
    d_ref, xw = ref.pm_density(x, n, wrap=True)
    d_ref = np.ascontiguousarray(d_ref[:, :, :n])
    fs.pm.init(n, 2.0, L)
    fs.pm.set_deposit_mode(mode)
    try:
        p = _particles(fs, L, x=x)
        p.set_a(1.0, 1.0, 0.0)
        fs.pm.send_positions(p)
        assert np.array_equal(p.x, xw)
        d = fs.pm.compute_density(p).asarray()
        fs.pm.compute_force(p)
        f = p.force
    finally:
        fs.pm.set_deposit_mode("atomic")
    assert rel_l2(d, d_ref) <= 1e-5
    assert np.abs(d - d_ref).max() < 500 * np.finfo(np.float32).eps * \
        max(1.0, float(np.abs(d_ref).max()))
    f_ref = ref.pm_force(xw, n, wrap=False)[0]
    print("\n%s vs reference: density %.2e, force %.2e"
          % (mode, rel_l2(d, d_ref), rel_l2(f, f_ref)))
    assert rel_l2(f, f_ref) <= 1e-4


def test_kick_drift_velocity_against_reference(fs, ref):
    # bit for bit: the GPU's kernels and the reference's loops on the same
    # particles (each with its own FP64 coefficients)
    rng = np.random.default_rng(13)
    N, L = 20001, 100.0
    x = rng.uniform(0, L, (N, 3)).astype(np.float32)
    v, d1, d2, f = (rng.standard_normal((N, 3)).astype(np.float32)
                    for _ in range(4))
    a_x, a_v, a_vel, a_pos = 0.3, 0.25, 0.35, 0.4
    p = _particles(fs, L, x=x, v=v, dx1=d1, dx2=d2, f=f)
    p.set_a(a_x, a_v, a_x)
    fs.cola.kick(p, a_vel)
    v_ref = ref.cola_kick(v, f, d1, d2, a_x, a_v, a_vel)
    assert np.array_equal(p.v, v_ref)
    fs.cola.drift(p, a_pos)
    x_ref = ref.cola_drift(x, v_ref, d1, d2, a_x, a_vel, a_pos)
    assert np.array_equal(p.x, x_ref)
    assert np.array_equal(fs.cola.velocity(p),
                          ref.cola_velocity(v_ref, d1, d2, a_pos))


def test_lpt_against_reference(fs, ref, eh_table):
    nc, L, a = 32, 64.0, 0.5
    x, v, d1, d2, ids, up, ua, _ = ref.lpt(nc, L, a, 5, eh_table, "2lpt")
    p = fs.lpt.init_from_draws(nc, L, a, fs.PowerSpectrum(eh_table), up, ua,
                               "2lpt")
    assert np.array_equal(p.id, ids)
    assert rel_l2(p.dx1, d1) <= 1e-5
    assert rel_l2(p.dx2, d2) <= 1e-4
    assert rel_l2(p.v, v) <= 1e-4
    assert np.abs(p.x - x).max() < 1e-4 * L / nc
