"""The oracle pinned to the reference's own code.

oracle/_ref/libfs2ref.so is the reference's py/pm.cpp, cola.cpp, lpt.cpp,
fft.cpp, cosmology.cpp, power.cpp (and the small files they need) compiled
from its sources with single-rank stand-ins for MPI, FFTW and GSL
(oracle/ref.py).  These tests run the same inputs through it and through
the oracle's restatement:

* bit for bit where no third-party arithmetic is involved -- the CIC
  deposit, the k-space force loop, the gather, kick, drift and
  cola_velocity;
* within float rounding where an FFT sits between (the stand-in FFT is
  double precision, the oracle's is pocketfft in float32): the full force
  and the 2LPT particles;
* the seed table's fill order (py/lpt.cpp:235-273), from the seeds the
  reference's code reseeded each column with.

No GPU.  Skipped where neither the reference sources nor a prebuilt
libfs2ref.so exist.
"""
import numpy as np
import pytest

OMEGA_M = 0.31


@pytest.fixture(scope="module")
def ref():
    import ref as R
    if R.lib() is None:
        pytest.skip("reference sources and oracle/_ref build both absent")
    R.init(OMEGA_M)
    return R


def _clustered(n_side, L, seed):
    rng = np.random.default_rng(seed)
    g = (np.stack(np.meshgrid(*[np.arange(n_side)] * 3, indexing="ij"), -1)
         .reshape(-1, 3) + 0.5) * (L / n_side)
    x = g + rng.normal(0, 0.6 * L / n_side, g.shape)
    clump = rng.normal(0.3 * L, 0.01 * L, (len(x) // 8, 3))
    x[: len(clump)] = clump
    # some positions outside the box, for the wrap
    x[-7:] = rng.uniform(-0.4 * L, 1.4 * L, (7, 3))
    return x.astype(np.float32)


def test_deposit_and_wrap_bitwise(ref, oracle_mod):
    n, L = 32, 32.0
    x = _clustered(16, L, 1)
    ref.pm_init(n, 2.0, L)
    d_ref, xw_ref = ref.pm_density(x, n, wrap=True)
    xw = oracle_mod.wrap(x.copy(), L)
    assert np.array_equal(xw, xw_ref)
    pm = oracle_mod.PM(n, 2.0, L, nthreads=1)
    d_or = pm.density(xw)
    assert np.array_equal(oracle_mod.unpad(d_or), oracle_mod.unpad(d_ref))


def test_kspace_force_and_gather_bitwise(ref, oracle_mod):
    n, L = 32, 32.0
    x = oracle_mod.wrap(_clustered(16, L, 2), L)
    ref.pm_init(n, 2.0, L)
    rng = np.random.default_rng(3)
    nk = n // 2 + 1
    dk = (rng.standard_normal((n, n, nk)) +
          1j * rng.standard_normal((n, n, nk))).astype(np.complex64)
    meshes = rng.standard_normal((3, n, n, 2 * nk)).astype(np.float32)
    f_ref, fk_ref, _, _ = ref.pm_force(x, n, wrap=False, dk_inject=dk,
                                    capture=True, mesh_inject=meshes)
    Lo = oracle_mod.lib()
    P = oracle_mod._p32
    f_or = np.zeros_like(x)
    for axis in range(3):
        fk = np.empty_like(dk)
        Lo.or_force_mesh_k(P(oracle_mod.cview(dk)), P(oracle_mod.cview(fk)),
                           n, np.float32(L), axis, 1)
        assert np.array_equal(fk.view(np.float32),
                              fk_ref[axis].view(np.float32)), axis
        Lo.or_force_gather(P(x), len(x), P(np.ascontiguousarray(meshes[axis])),
                           n, np.float32(L), axis, P(f_or), 1)
    assert np.array_equal(f_or, f_ref)


def test_full_force_within_fft_rounding(ref, oracle_mod):
    n, L = 32, 32.0
    x = oracle_mod.wrap(_clustered(16, L, 4), L)
    ref.pm_init(n, 2.0, L)
    f_ref, fk_ref, meshes_ref, _ = ref.pm_force(x, n, wrap=False, capture=True)
    pm = oracle_mod.PM(n, 2.0, L, nthreads=1)
    pm.density(x)
    f_or = pm.force(x)
    rel = np.linalg.norm(f_or - f_ref) / np.linalg.norm(f_ref)
    assert rel < 1e-5, rel
    for a in range(3):
        m_or = oracle_mod.unpad(pm.force_meshes[a])
        m_ref = oracle_mod.unpad(meshes_ref[a])
        assert np.linalg.norm(m_or - m_ref) / np.linalg.norm(m_ref) < 1e-5


def test_kick_drift_velocity_bitwise(ref, oracle_mod):
    rng = np.random.default_rng(5)
    N = 5000
    x = rng.uniform(0, 100.0, (N, 3)).astype(np.float32)
    v, d1, d2, f = (rng.standard_normal((N, 3)).astype(np.float32)
                    for _ in range(4))
    a_x, a_v, a_vel, a_pos = 0.3, 0.25, 0.35, 0.4
    cosmo = oracle_mod.Cosmology(OMEGA_M)
    st = oracle_mod.ParticleState(x.copy(), v.copy(), d1, d2,
                                  np.zeros(N, np.uint64), a_x=a_x, a_v=a_v,
                                  f=f)
    v_ref = ref.cola_kick(v, f, d1, d2, a_x, a_v, a_vel)
    oracle_mod.cola_kick(st, cosmo, a_vel)
    assert np.array_equal(st.v, v_ref)
    x_ref = ref.cola_drift(x, v_ref, d1, d2, a_x, a_vel, a_pos)
    oracle_mod.cola_drift(st, cosmo, a_pos)
    assert np.array_equal(st.x, x_ref)
    u_ref = ref.cola_velocity(st.v, d1, d2, a_pos)
    assert np.array_equal(oracle_mod.cola_velocity(st, cosmo), u_ref)


def test_growth_coefficients_agree(ref, oracle_mod):
    # the reference's cosmology (with the stand-in quadrature) and the
    # oracle's FP64 functions, to 1e-12 relative
    L = ref.lib()
    cosmo = oracle_mod.Cosmology(OMEGA_M)
    for a in (0.02, 0.1, 0.37, 0.5, 1.0):
        D = L.fs2ref_D_growth(a)
        assert abs(D / cosmo.D(a) - 1) < 1e-12
        assert abs(L.fs2ref_D2_growth(a, D) / cosmo.D2(a, D) - 1) < 1e-12
        assert abs(L.fs2ref_Dv_growth(a, D) / cosmo.Dv(a, D) - 1) < 1e-12


@pytest.mark.parametrize("kind", ["cola", "2lpt", "zeldovich"])
def test_lpt_from_the_references_draws(ref, oracle_mod, eh_table, kind):
    # the reference's 2LPT with the logged stand-in stream, and the oracle
    # fed the very draws each mode received
    nc, L, a = 16, 32.0, 0.5
    x, v, d1, d2, ids, up, ua, _ = ref.lpt(nc, L, a, 7, eh_table, kind)
    q = oracle_mod.lpt(nc, L, a, up, ua, oracle_mod.PowerSpectrum(eh_table),
                       oracle_mod.Cosmology(OMEGA_M), kind)
    assert np.array_equal(q.id, ids)
    rel = lambda s, t: np.linalg.norm(s - t) / np.linalg.norm(t)
    assert rel(q.dx1, d1) < 1e-5
    assert rel(q.dx2, d2) < 1e-5
    assert np.abs(q.x - x).max() < 1e-5 * L / nc
    if kind == "cola":
        assert np.all(v == 0) and np.all(q.v == 0)
    else:
        assert rel(q.v, v) < 1e-5


def test_seed_table_order(ref, oracle_mod, eh_table):
    # py/lpt.cpp:235-273 (N-GenIC): the first nc^2 draws fill the table in
    # a symmetric spiral; column (ix, iy) is then reseeded with
    # table[ix*nc + iy] (:319).  The oracle's restatement of the fill
    # order, fed the same first nc^2 draws, gives the seeds the reference's
    # code used.
    nc = 16
    *_, seeds = ref.lpt(nc, 32.0, 0.5, 11, eh_table, "cola")
    L = ref.lib()
    import ctypes
    m = L.fs2ref_rng_log_size()
    u = np.zeros(m, np.float64)
    s = np.zeros(m, np.uint64)
    L.fs2ref_rng_log_copy(s.ctypes.data_as(ctypes.POINTER(ctypes.c_ulong)),
                          u.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    table = oracle_mod.seedtable(nc, u[: nc * nc])
    used = seeds[nc * nc:].reshape(nc, nc, nc)[:, :, 0]
    assert np.array_equal(table.reshape(nc, nc).astype(np.uint64), used)


def _golden():
    import os
    here = os.path.dirname(os.path.abspath(__file__))
    return np.load(os.path.join(here, "golden", "ref_cola_16p_32m.npz"))


def test_reference_fixture_is_current(ref):
    # the committed fixture is what the compiled reference computes now
    import os
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.join(here, "golden"))
    import make_ref_golden
    g = _golden()
    out = make_ref_golden.run()
    ref.init(OMEGA_M)
    for k in ("u_phase", "u_ampl", "x0", "dx1", "dx2", "delta0", "f0", "x",
              "v"):
        assert np.array_equal(out[k], g[k]), k


def test_oracle_reproduces_reference_fixture(oracle_mod, eh_table):
    # the oracle, fed the draws the reference's run used, through the same
    # 2LPT + 3 COLA steps: the same numbers within the FFTs' float rounding
    # (needs only the committed fixture, not the reference sources)
    from fs2_b200 import power_eh
    g = _golden()
    nc, n, L = int(g["case_nc"]), int(g["case_n"]), float(g["case_boxsize"])
    a0, a1, ns = (float(g["case_a_init"]), float(g["case_a_final"]),
                  int(g["case_nstep"]))
    k, P = power_eh.eh_nowiggle_table()
    cosmo = oracle_mod.Cosmology(float(g["case_omega_m"]))
    p = oracle_mod.lpt(nc, L, a0, g["u_phase"], g["u_ampl"],
                       oracle_mod.PowerSpectrum(eh_table), cosmo, "cola")
    rel = lambda s, t: np.linalg.norm(s - t) / np.linalg.norm(t)
    assert np.array_equal(p.id, g["id"])
    assert rel(p.dx1, g["dx1"]) < 1e-5 and rel(p.dx2, g["dx2"]) < 1e-5
    pm = oracle_mod.PM(n, n / nc, L)
    for i in range(ns):
        a_vel = a0 + (a1 - a0) / ns * (i + 0.5)
        oracle_mod.pm_force(p, pm)
        if i == 0:
            assert rel(p.f, g["f0"]) < 1e-5
        oracle_mod.cola_kick(p, cosmo, a_vel)
        oracle_mod.cola_drift(p, cosmo, a0 + (a1 - a0) / ns * (i + 1.0))
    d = p.x.astype(np.float64) - g["x"]
    d -= L * np.round(d / L)
    assert np.sqrt(np.mean(d ** 2)) < 1e-4 * L / n
    assert rel(p.v, g["v"]) < 1e-5
