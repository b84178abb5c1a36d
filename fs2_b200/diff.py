"""Differentiable COLA with torch.autograd.

    sim = DifferentiableCOLA(nc=128, n=256, boxsize=128.0, pk_table=path,
                             a_init=0.1, a_final=1.0, nsteps=10)
    w = torch.randn(128, 128, 128, device="cuda", requires_grad=True)
    delta = sim(w)                       # final CIC density contrast, (n,n,n)
    loss = ((delta - target) ** 2).mean()
    loss.backward()                      # w.grad by the hand-written adjoint

Forward and backward run in libfs2gpu (fs2g_diff_forward / _backward): the
white noise is turned into delta(k) = T(k) FFT(w) with T = sqrt(P/(V nc^3)),
2LPT particles at a_init, nsteps COLA steps on the schedule of the
reference's driver (script/cola.py:37-44), and the CIC density of the final
positions.  The backward applies the transposed stages in reverse with
per-step checkpointing.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import capi


def cola_schedule(a_init, a_final, nsteps):
    """(a_vel, a_pos) arrays of script/cola.py:37-44."""
    da = (a_final - a_init) / nsteps
    a_vel = np.array([a_init + da * (i + 0.5) for i in range(nsteps)])
    a_pos = np.array([a_init + da * (i + 1.0) for i in range(nsteps)])
    return a_vel, a_pos


class DifferentiableCOLA:
    def __init__(self, nc, n, boxsize, pk_table, a_init, a_final, nsteps,
                 omega_m=0.31):
        import fs2_b200.fs as fs
        self.fs = fs
        fs.cosmology.init(omega_m)
        self.nc, self.n, self.boxsize = nc, n, boxsize
        self._ps = C.c_void_p()
        capi.call("fs2g_power_alloc", str(pk_table).encode(),
                  C.byref(self._ps))
        self.a_vel, self.a_pos = cola_schedule(a_init, a_final, nsteps)
        av = np.ascontiguousarray(self.a_vel, dtype=np.float64)
        ap = np.ascontiguousarray(self.a_pos, dtype=np.float64)
        self._d = C.c_void_p()
        capi.call("fs2g_diff_create", C.c_void_p(fs._fs._ctx_address()), nc, n,
                  float(boxsize), self._ps, float(a_init), nsteps,
                  capi.dptr(av), capi.dptr(ap), C.byref(self._d))

    def close(self):
        if self._d:
            capi.lib().fs2g_diff_free(self._d)
            self._d = C.c_void_p()
        if self._ps:
            capi.lib().fs2g_power_free(self._ps)
            self._ps = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check_w(self, w):
        if not (w.is_cuda and w.dtype == torch.float32):
            raise TypeError("white noise must be a float32 CUDA tensor")
        if tuple(w.shape) != (self.nc,) * 3:
            raise ValueError("white noise must have shape (nc, nc, nc)")

    def forward_raw(self, w):
        """Final density (n, n, n) for white noise w (no autograd)."""
        self._check_w(w)
        w = w.contiguous()
        out = torch.empty((self.n,) * 3, dtype=torch.float32, device=w.device)
        torch.cuda.current_stream().synchronize()
        capi.call("fs2g_diff_forward", self._d, C.c_void_p(w.data_ptr()),
                  C.c_void_p(out.data_ptr()))
        self.fs._fs._synchronize()
        return out

    def backward_raw(self, delta_bar):
        """dL/dw for dL/d(final density) = delta_bar, after forward_raw."""
        delta_bar = delta_bar.contiguous().to(torch.float32)
        wbar = torch.empty((self.nc,) * 3, dtype=torch.float32,
                           device=delta_bar.device)
        torch.cuda.current_stream().synchronize()
        capi.call("fs2g_diff_backward", self._d,
                  C.c_void_p(delta_bar.data_ptr()), C.c_void_p(wbar.data_ptr()))
        self.fs._fs._synchronize()
        return wbar

    def __call__(self, w):
        return _COLAFunction.apply(w, self)


class _COLAFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, w, sim):
        ctx.sim = sim
        return sim.forward_raw(w)

    @staticmethod
    def backward(ctx, g):
        return ctx.sim.backward_raw(g), None
