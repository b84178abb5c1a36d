"""The differentiable COLA run (fs2_b200/diff.py): forward against a float64
torch restatement (oracle/diff_torch.py), the hand-written adjoint against
that restatement's autograd gradient, and against central finite
differences.

CIC weights are piecewise linear in position, so the exact gradient of a
density loss jumps wherever a particle crosses a mesh plane: it is defined
almost everywhere but is rough.  At 128^3/256^3 after 10 steps the float64
restatement's own gradient moves by ~2e-2 (relative L2) when the noise
moves by 1e-5 of its norm, and its central differences with eps = 1e-3
along random unit directions differ from its own exact directional
derivatives by ~1.5e-3 (the error of a central difference across kinks
grows linearly with eps).  Float32 positions carry rounding of ~1e-5 cell,
which puts a few particles on the other side of a plane from the float64
trajectory, so the full-vector difference of the float32 and float64
gradients is set by that roughness, not by the adjoint's arithmetic.  The
tests therefore check
  * quantities that are smooth: the float32 gradient's projection on the
    float64 gradient, and the central difference (eps = 1e-4) along the
    gradient direction, each to 1e-3;
  * the full vectors against the oracle's own roughness under a nudge of
    the noise of 1e-5 of its norm (position changes just above float32
    rounding);
  * the 16 random-direction differences (eps = 1e-3) against the float64
    adjoint's own finite-difference error plus the full-vector difference.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

OMEGA_M = 0.31


def _rel(a, b):
    a = a.double().flatten()
    b = b.double().flatten()
    return float((a - b).norm() / b.norm())


@pytest.fixture(scope="module")
def ps_oracle(oracle_mod, eh_table):
    return oracle_mod.PowerSpectrum(eh_table)


def _sim(eh_table, nc, n, L, a0, a1, ns):
    from fs2_b200.diff import DifferentiableCOLA
    return DifferentiableCOLA(nc, n, L, eh_table, a0, a1, ns, OMEGA_M)


def _noise(nc, seed, device="cuda"):
    g = torch.Generator().manual_seed(seed)
    return torch.randn((nc,) * 3, generator=g, dtype=torch.float64).to(device)


def test_small_forward_and_gradient_vs_fp64(eh_table, ps_oracle):
    import diff_torch
    import fs2_b200.fs as fs
    nc, n, L, a0, a1, ns = 16, 32, 32.0, 0.1, 0.6, 3
    sim = _sim(eh_table, nc, n, L, a0, a1, ns)
    fs.pm.set_deposit_mode("deterministic")
    try:
        w64 = _noise(nc, 2, "cpu")
        t = (_noise(n, 3, "cpu") * 0.3).float()
        w = w64.float().cuda().requires_grad_(True)
        delta = sim(w)
        loss = ((delta.double() - t.cuda().double()) ** 2).mean()
        loss.backward()
        g_gpu = w.grad.detach().cpu()
    finally:
        fs.pm.set_deposit_mode("atomic")
    wr = w64.clone().requires_grad_(True)
    d64 = diff_torch.run(wr, nc, n, L, a0, sim.a_vel, sim.a_pos, ps_oracle,
                         OMEGA_M)
    l64 = ((d64 - t.double()) ** 2).mean()
    l64.backward()
    assert _rel(delta.detach().cpu(), d64.detach()) <= 1e-4
    assert _rel(g_gpu, wr.grad) <= 1e-3
    sim.close()


def test_config4_gradient_fp64_and_finite_differences(eh_table, ps_oracle):
    # 128^3 particles, 256^3 mesh, 128 Mpc/h, white noise seed 2, 10 COLA
    # steps from a = 0.1 to 1; loss = mean((delta - delta[seed 3])^2)
    import diff_torch
    nc, n, L, a0, a1, ns = 128, 256, 128.0, 0.1, 1.0, 10
    sim = _sim(eh_table, nc, n, L, a0, a1, ns)
    target = sim.forward_raw(_noise(nc, 3).float()).double()
    w = _noise(nc, 2).float().requires_grad_(True)
    delta = sim(w)
    loss = ((delta.double() - target) ** 2).mean()
    loss.backward()
    g = w.grad.detach().double()

    def run64(w_):
        return diff_torch.run(w_, nc, n, L, a0, sim.a_vel, sim.a_pos,
                              ps_oracle, OMEGA_M)

    def loss64(w_):
        return ((run64(w_) - target) ** 2).mean()

    def grad64(w_):
        w_ = w_.clone().requires_grad_(True)
        loss64(w_).backward()
        return w_.grad.detach()

    w64 = _noise(nc, 2)
    g64 = grad64(w64)
    # roughness of the exact gradient under small nudges of the noise
    rough = {eta: _rel(grad64(w64 + eta * _noise(nc, 11)), g64)
             for eta in (1e-6, 1e-5)}
    rel_grad = _rel(g, g64)
    proj = float((g * g64).sum() / (g64 * g64).sum())

    def central(u, eps):
        with torch.no_grad():
            return float((loss64(w64 + eps * u) - loss64(w64 - eps * u))
                         / (2 * eps))

    # along the gradient direction (eps = 1e-4) ...
    u0 = g64 / g64.norm()
    fd0 = central(u0, 1e-4)
    rel_fd_grad_dir = abs(fd0 - float((g * u0).sum())) / abs(fd0)
    # ... and along 16 random unit directions, eps = 1e-3
    gen = torch.Generator().manual_seed(7)
    fd, ad, ad64 = [], [], []
    for _ in range(16):
        u = torch.randn((nc,) * 3, generator=gen, dtype=torch.float64).cuda()
        u /= u.norm()
        fd.append(central(u, 1e-3))
        ad.append(float((g * u).sum()))
        ad64.append(float((g64 * u).sum()))
    fd, ad, ad64 = np.array(fd), np.array(ad), np.array(ad64)
    rel_fd = float(np.linalg.norm(fd - ad) / np.linalg.norm(fd))
    rel_fd64 = float(np.linalg.norm(fd - ad64) / np.linalg.norm(fd))
    print("config4: |g-g64|/|g64| %.2e (g64 roughness %.2e at 1e-6, %.2e at "
          "1e-5), projection-1 %.2e, FD along g64 %.2e, FD 16 random dirs "
          "%.2e (float64 adjoint %.2e)"
          % (rel_grad, rough[1e-6], rough[1e-5], proj - 1, rel_fd_grad_dir,
             rel_fd, rel_fd64))
    assert abs(proj - 1) <= 1e-3
    assert rel_fd_grad_dir <= 1e-3
    assert rel_grad <= rough[1e-5]
    assert rel_fd <= rel_fd64 + 1.5 * rel_grad
    sim.close()


def test_force_checkpoints_equal_recomputation(eh_table):
    # the cuFFT engine keeps each step's force meshes from the forward; the
    # fused engine (forced at n = 64) recomputes them in the backward.  The
    # two gradients agree to the engines' FFT rounding.
    import fs2_b200.fs as fs
    nc, n, L, a0, a1, ns = 32, 64, 64.0, 0.1, 0.6, 3
    w0 = _noise(nc, 7).float()
    t = (_noise(n, 8) * 0.3).float()
    grads, losses = [], []
    fs.pm.set_deposit_mode("deterministic")
    try:
        for engine in ("cufft", "fused"):
            fs.pm.set_fft_engine(engine)
            fs.pm.free()
            sim = _sim(eh_table, nc, n, L, a0, a1, ns)
            try:
                assert fs.pm.fused() == (engine == "fused")
                w = w0.clone().requires_grad_(True)
                loss = ((sim(w).double() - t.double()) ** 2).mean()
                loss.backward()
                grads.append(w.grad.detach().double().cpu())
                losses.append(float(loss.detach()))
            finally:
                sim.close()
    finally:
        fs.pm.set_fft_engine("auto")
        fs.pm.set_deposit_mode("atomic")
        fs.pm.free()
    assert abs(losses[0] / losses[1] - 1) <= 1e-5
    assert _rel(grads[0], grads[1]) <= 1e-4
