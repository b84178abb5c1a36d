"""The batched ensemble (fs2_b200/ensemble.py, fs2g_ensemble_*): one CUDA
graph over members of uneven sizes against the members looped on one
stream, and against the single differentiable run of each member
(fs2_b200/diff.py).  With the deterministic deposit the forward (density,
loss) is bit for bit the same every way; the backward's scatters use float
atomics, so gradients agree to rounding (relative L2 <= 1e-5)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

OMEGA_M = 0.31
A0, A1, NSTEPS = 0.1, 0.5, 2


@pytest.fixture(scope="module")
def fs():
    import fs2_b200.fs as fs
    fs.cosmology.init(OMEGA_M)
    return fs


def _members():
    from fs2_b200.ensemble import Member
    # one size twice, a size the fused pipeline cannot do (n = 48) and a
    # larger one
    return [Member(16, 32, 32.0, 100), Member(16, 32, 32.0, 101),
            Member(24, 48, 48.0, 102), Member(32, 64, 32.0, 103)]


def _rel(a, b):
    a, b = a.double().flatten(), b.double().flatten()
    return float((a - b).norm() / b.norm())


def _noise(side, seed):
    g = torch.Generator().manual_seed(seed)
    return torch.randn((side,) * 3, generator=g).cuda()


@pytest.fixture()
def deterministic(fs):
    fs.pm.set_deposit_mode("deterministic")
    yield
    fs.pm.set_deposit_mode("atomic")


def _build(eh_table, autotune):
    from fs2_b200.ensemble import Ensemble
    mem = _members()
    ens = Ensemble(mem, eh_table, A0, A1, NSTEPS, OMEGA_M, autotune=autotune)
    for i, m in enumerate(mem):
        ens.set_noise(i, _noise(m.nc, m.seed + 1000))
        t = ens.forward_member(i).clone()
        ens.set_target(i, t)
        ens.set_noise(i, _noise(m.nc, m.seed))
    return mem, ens


def test_graph_equals_loop_and_single_runs(fs, eh_table, deterministic):
    from fs2_b200.diff import DifferentiableCOLA
    mem, ens = _build(eh_table, autotune=False)
    try:
        ens.run(graph=False)
        loss_loop = ens.losses()
        grad_loop = [ens.gradient(i).clone() for i in range(len(mem))]
        for rep in range(2):                 # capture, then replay
            ens.run(graph=True)
            loss_graph = ens.losses()
            assert np.array_equal(loss_graph, loss_loop)
            for i in range(len(mem)):
                assert _rel(ens.gradient(i), grad_loop[i]) <= 1e-5
        # each member against its own single differentiable run
        for i, m in enumerate(mem):
            sim = DifferentiableCOLA(m.nc, m.n, m.boxsize, eh_table, A0, A1,
                                     NSTEPS, OMEGA_M)
            try:
                delta = sim.forward_raw(_noise(m.nc, m.seed))
                d = delta - ens.target(i)
                inv = np.float32(1.0) / np.float32(m.n ** 3)
                dbar = 2.0 * d * float(inv)
                wbar = sim.backward_raw(dbar)
            finally:
                sim.close()
            assert torch.equal(delta, ens.density(i))
            assert _rel(wbar, grad_loop[i]) <= 1e-5
            ref = float((d.double() ** 2).mean())
            assert abs(loss_loop[i] - ref) <= 1e-12 * max(ref, 1e-30)
            assert loss_loop[i] > 0
    finally:
        ens.close()


def test_autotuner_choices(fs, eh_table):
    mem, ens = _build(eh_table, autotune=True)
    try:
        tun = ens.tuning()
        for m, (engine, tile, ms) in zip(mem, tun):
            assert ms > 0
            assert tile in (4, 8)
            if m.n == 48:
                assert engine == "cufft"        # no fused pipeline for 48
        # members of one size share the choice
        assert tun[0] == tun[1]
        ens.run(graph=True)
        assert np.all(np.isfinite(ens.losses()))
    finally:
        ens.close()
