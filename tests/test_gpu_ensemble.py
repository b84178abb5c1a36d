"""The batched ensemble (fs2_b200/ensemble.py, fs2g_ensemble_*): size
classes run as batched chunks in one CUDA graph, against the members looped
one by one through the unbatched path, and against the single
differentiable run of each member (fs2_b200/diff.py).  With the
deterministic deposit a graph replay is bit for bit the previous one, and
the loop mode bit for bit the single runs.  Batched and unbatched runs do
the same arithmetic per member except inside cuFFT, whose batched plans may
order a transform's operations differently: density and loss agree to
float rounding (relative 1e-6), gradients to relative L2 <= 1e-5 (the
backward's scatters use float atomics)."""
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
        dens_loop = [ens.density(i).clone() for i in range(len(mem))]
        grad_loop = [ens.gradient(i).clone() for i in range(len(mem))]
        loss_first = None
        for rep in range(2):                 # capture, then replay
            ens.run(graph=True)
            loss_graph = ens.losses()
            if loss_first is None:
                loss_first = loss_graph
            assert np.array_equal(loss_graph, loss_first)
            assert np.allclose(loss_graph, loss_loop, rtol=1e-6, atol=0)
            for i in range(len(mem)):
                assert _rel(ens.density(i), dens_loop[i]) <= 1e-6
                assert _rel(ens.gradient(i), grad_loop[i]) <= 1e-5
        # the graph holds one chunk per size class: a few hundred kernels,
        # not one set per member
        assert 0 < ens.graph_kernels() < 1000
        ens.run(graph=False)
        assert np.array_equal(ens.losses(), loss_loop)
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
            assert torch.equal(delta, dens_loop[i])
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
        sizes = {}
        for m in mem:
            sizes[(m.nc, m.n, m.boxsize)] = sizes.get((m.nc, m.n, m.boxsize), 0) + 1
        for m, (engine, chunk, ms) in zip(mem, tun):
            B = sizes[(m.nc, m.n, m.boxsize)]
            assert ms > 0
            assert chunk in {(B + d - 1) // d for d in (1, 2, 4)}
            assert engine == "cufft"            # batched plans
        # members of one size share the choice
        assert tun[0] == tun[1]
        ens.run(graph=True)
        assert np.all(np.isfinite(ens.losses()))
    finally:
        ens.close()


def test_batched_chunks_match_loop(fs, eh_table):
    # atomic deposit, a class of three members split into chunks of 2 + 1
    # by the tuner's candidates: every chunk split gives the loop's losses
    # to float rounding
    from fs2_b200.ensemble import Ensemble, Member
    mem = [Member(16, 32, 32.0, 200 + k) for k in range(3)]
    ens = Ensemble(mem, eh_table, A0, A1, NSTEPS, OMEGA_M, autotune=True)
    try:
        for i, m in enumerate(mem):
            ens.set_noise(i, _noise(m.nc, m.seed + 1000))
            ens.set_target(i, ens.forward_member(i).clone())
            ens.set_noise(i, _noise(m.nc, m.seed))
        ens.run(graph=False)
        loss_loop = ens.losses()
        ens.run(graph=True)
        assert np.allclose(ens.losses(), loss_loop, rtol=1e-5, atol=0)
        assert np.all(loss_loop > 0)
    finally:
        ens.close()
