"""FP64 reference gradient for the differentiable COLA run.

TEST INFRASTRUCTURE ONLY (the oracle of fs2_b200/diff.py): the same forward
model written with torch operations in float64 on the CPU -- pocketfft
transforms (whose C2R takes the real part on the kz = 0 and n/2 planes, like
the GPU path), CIC deposit by index_add_, CIC gather by indexing, the
reference's kick and drift -- so that torch.autograd gives an independent
gradient with respect to the white-noise field.  The reference (fs2) has no
gradients; the loops it restates are py/lpt.cpp:465-586 (2LPT), py/pm.cpp
(deposit, force, gather) and py/cola.cpp:48-127 (kick, drift).
"""
import math

import numpy as np
import torch

import oracle


def _lpt_k(nc, boxsize, device="cpu"):
    dk = 2 * math.pi / boxsize
    i = torch.arange(nc, dtype=torch.float64, device=device)
    k = torch.where(i < nc // 2, dk * i, -dk * (nc - i))
    kz = k[: nc // 2 + 1]
    return torch.meshgrid(k, k, kz, indexing="ij")


def _transfer(nc, boxsize, ps, device="cpu"):
    K = _lpt_k(nc, boxsize, device)
    k2 = K[0] ** 2 + K[1] ** 2 + K[2] ** 2
    kk = torch.sqrt(k2).cpu().numpy().copy()
    kk[0, 0, 0] = 1.0
    P = torch.from_numpy(ps.P(kk)).to(device)
    T = torch.sqrt(P / (boxsize ** 3 * nc ** 3))
    T[0, 0, 0] = 0
    T[nc // 2] = 0
    T[:, nc // 2] = 0
    T[:, :, nc // 2] = 0
    return T, K, k2


def lpt(w, boxsize, a, ps, cosmo):
    nc = w.shape[0]
    dev = w.device
    T, K, k2 = _transfer(nc, boxsize, ps, dev)
    k2s = k2.clone()
    k2s[0, 0, 0] = 1.0
    X = torch.fft.rfftn(w)
    dk = T * X
    s = (nc, nc, nc)
    irf = lambda z: torch.fft.irfftn(z, s=s, norm="forward")
    psi_k = [1j * K[i] / k2s * dk for i in range(3)]
    ij = [(0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2)]
    p = [irf(1j * K[j] * psi_k[i]) for i, j in ij]
    S = p[0] * (p[3] + p[5]) + p[3] * p[5] - p[1] ** 2 - p[2] ** 2 - p[4] ** 2
    Sk = torch.fft.rfftn(S)
    psi2_k = [-1j * K[i] / k2s * Sk for i in range(3)]
    for q in psi2_k:
        q[0, 0, 0] = 0
    psi = torch.stack([irf(q) for q in psi_k], -1).reshape(-1, 3)
    psi2 = torch.stack([irf(q) for q in psi2_k], -1).reshape(-1, 3) / nc ** 3
    D1 = cosmo.D(a)
    D2 = cosmo.D2(a, D1)
    g = torch.arange(nc, dtype=torch.float64, device=dev)
    q = torch.stack(torch.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    q = (q + 0.5) * (boxsize / nc)
    x = q + D1 * psi + D2 * psi2
    return x, psi, psi2


def _cic(x, n, boxsize):
    X = x * (n / boxsize)
    i0 = torch.floor(X.detach())
    w1 = X - i0
    w0 = 1 - w1
    i0 = i0.long() % n
    i1 = (i0 + 1) % n
    return i0, i1, w0, w1


def _corners(i0, i1, w0, w1, n):
    for o in range(8):
        ix = i1[:, 0] if o & 4 else i0[:, 0]
        iy = i1[:, 1] if o & 2 else i0[:, 1]
        iz = i1[:, 2] if o & 1 else i0[:, 2]
        w = ((w1[:, 0] if o & 4 else w0[:, 0]) * (w1[:, 1] if o & 2 else w0[:, 1])
             * (w1[:, 2] if o & 1 else w0[:, 2]))
        yield (ix * n + iy) * n + iz, w


def density(x, n, boxsize, fac):
    i0, i1, w0, w1 = _cic(x, n, boxsize)
    m = torch.zeros(n ** 3, dtype=torch.float64, device=x.device)
    for idx, w in _corners(i0, i1, w0, w1, n):
        m = m.index_add(0, idx, fac * w)
    return m.reshape(n, n, n) - 1.0


def force(x, n, boxsize, fac):
    d = density(x, n, boxsize, fac)
    dk = torch.fft.rfftn(d)
    i = torch.arange(n, dtype=torch.float64, device=x.device)
    k = torch.where(i <= n // 2, i, i - n)
    kz = torch.arange(n // 2 + 1, dtype=torch.float64, device=x.device)
    K = torch.meshgrid(k, k, kz, indexing="ij")
    k2 = K[0] ** 2 + K[1] ** 2 + K[2] ** 2
    k2[0, 0, 0] = 1.0
    f1 = -1.0 / n ** 3 / (2 * math.pi / boxsize)
    i0, i1, w0, w1 = _cic(x, n, boxsize)
    out = []
    for a in range(3):
        fk = 1j * f1 * K[a] / k2 * dk
        fk[0, 0, 0] = 0
        g = torch.fft.irfftn(fk, s=(n, n, n), norm="forward").reshape(-1)
        fa = 0
        for idx, w in _corners(i0, i1, w0, w1, n):
            fa = fa + w * g[idx]
        out.append(fa)
    return torch.stack(out, -1)


def wrap(x, boxsize):
    return x - boxsize * torch.floor(x.detach() / boxsize)


def run(w, nc, n, boxsize, a_init, a_vel, a_pos, ps, omega_m):
    """Final density for white noise w (float64 tensor (nc,nc,nc))."""
    cosmo = oracle.Cosmology(omega_m)
    fac = (n / nc) ** 3
    x, dx1, dx2 = lpt(w, boxsize, a_init, ps, cosmo)
    v = torch.zeros_like(x)
    a_x = a_v = a_init
    for av1, ap1 in zip(a_vel, a_pos):
        x = wrap(x, boxsize)
        f = force(x, n, boxsize, fac)
        om, kf, q1, q2 = oracle.kick_coefficients(cosmo, a_v, a_x, av1)
        v = v + float(kf) * (-1.5 * om) * (f + float(q1) * dx1 + float(q2) * dx2)
        a_v = av1
        dt, da1, da2 = oracle.drift_coefficients(cosmo, a_x, a_v, ap1)
        x = x + dt * v + float(da1) * dx1 + float(da2) * dx2
        a_x = ap1
    x = wrap(x, boxsize)
    return density(x, n, boxsize, fac)
