"""Batched uneven ensembles of differentiable COLA runs.

    members = config5_members()                 # 48 (nc, n, L, seed)
    mine = shard(members, world, rank)          # this rank's members
    ens = Ensemble(mine, pk_table, a_init=0.1, a_final=1.0, nsteps=5)
    ens.set_noise(i, w)        # (nc, nc, nc) float32 CUDA tensors
    ens.set_target(i, t)       # (n, n, n)
    ens.run(graph=True)        # forward, loss, backward of every member
    ens.losses()               # mean((delta - target)^2) per member
    ens.gradient(i)            # d loss / d noise, (nc, nc, nc)

The members run in libfs2gpu (fs2g_ensemble_*).  Members of one size
(nc, n, boxsize) form a class that runs in chunks; a chunk is one batched
differentiable run whose kernels and batched cuFFT transforms cover all of
its members at once.  graph=True replays every chunk as a single CUDA graph
(chunks side by side on their own streams); graph=False is the plain path,
looped: each member alone through its own unbatched run, one after another
on one stream.  The autotuner picks the members per chunk of each class.
Ranks take disjoint shards of the members; no data crosses between GPUs.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import capi
from .diff import cola_schedule


@dataclass(frozen=True)
class Member:
    nc: int          # particles per side
    n: int           # mesh cells per side
    boxsize: float   # Mpc/h
    seed: int        # white-noise seed


def config5_members():
    """48 realisations: 16 each of 32^3/64^3 (32 Mpc/h), 64^3/128^3
    (64 Mpc/h) and 96^3/192^3 (96 Mpc/h), seeds 100-147."""
    out = []
    seed = 100
    for nc, n, L in ((32, 64, 32.0), (64, 128, 64.0), (96, 192, 96.0)):
        for _ in range(16):
            out.append(Member(nc, n, L, seed))
            seed += 1
    return out


def step_bytes(m: Member) -> int:
    """Algorithmic HBM bytes of one COLA step of a member (the cost model
    of the sharding): 120 N + 32 n^3 + 32 n^2 (n/2 + 1)."""
    N, n = m.nc ** 3, m.n
    return 120 * N + 32 * n ** 3 + 32 * n * n * (n // 2 + 1)


def adjoint_step_bytes(m: Member) -> int:
    """Algorithmic HBM bytes of one step of a member's backward, with the
    forward's force meshes read from their checkpoints: restore x, v (48 N),
    fold x (24 N), the kick/drift transpose (96 N), the force cotangent
    scattered into three zeroed meshes (24 N + 12 R + 24 R), three R2C
    (12 R + 24 K), the Poisson adjoint (32 K), one C2R (4 R + 8 K) and the
    position adjoint's gather of four meshes (48 N + 16 R);
    N = nc^3, R = n^3, K = n^2 (n/2 + 1)."""
    N, n = m.nc ** 3, m.n
    R, K = n ** 3, n * n * (n // 2 + 1)
    return 240 * N + 68 * R + 64 * K


def lpt_bytes(m: Member) -> int:
    """Algorithmic HBM bytes of a member's 2LPT from white noise (psi(k),
    the six psi_ij, the source, psi2, 12 C2R + 1 R2C and the particle grid,
    232 K + 160 R at the particle grid's nc); its adjoint is counted as
    twice that."""
    nc = m.nc
    R, K = nc ** 3, nc * nc * (nc // 2 + 1)
    return 232 * K + 160 * R


def eval_bytes(m: Member, nsteps: int) -> int:
    """Algorithmic HBM bytes of one ensemble evaluation of a member:
    2LPT, nsteps forward steps, the loss, nsteps backward steps and the
    2LPT adjoint."""
    n = m.n
    return (nsteps * (step_bytes(m) + adjoint_step_bytes(m)) +
            3 * lpt_bytes(m) + 16 * n ** 3)


def shard(members, world, rank):
    """Members of `rank` under greedy longest-first balancing of
    step_bytes over `world` ranks (each member goes to the least-loaded
    rank; ties to the lower rank).  Every rank computes the same
    assignment, so no communication is needed."""
    return [members[i] for i in assignment(members, world)[rank]]


def assignment(members, world):
    """Indices of the members on each rank (see shard)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(members)),
                   key=lambda i: (-step_bytes(members[i]), i))
    load = [0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += step_bytes(members[i])
    return [sorted(p) for p in parts]


class _Dev:
    def __init__(self, ptr, shape):
        self.__cuda_array_interface__ = {
            "shape": shape, "typestr": "<f4", "data": (ptr, False),
            "version": 3}


class Ensemble:
    def __init__(self, members, pk_table, a_init, a_final, nsteps,
                 omega_m=0.31, autotune=True):
        import fs2_b200.fs as fs
        fs.cosmology.init(omega_m)
        self.members = list(members)
        self.a_vel, self.a_pos = cola_schedule(a_init, a_final, nsteps)
        self._ps = C.c_void_p()
        capi.call("fs2g_power_alloc", str(pk_table).encode(),
                  C.byref(self._ps))
        k = len(self.members)
        nc = (C.c_int * k)(*[m.nc for m in self.members])
        n = (C.c_int * k)(*[m.n for m in self.members])
        L = (C.c_double * k)(*[m.boxsize for m in self.members])
        av = np.ascontiguousarray(self.a_vel, dtype=np.float64)
        ap = np.ascontiguousarray(self.a_pos, dtype=np.float64)
        self._e = C.c_void_p()
        capi.call("fs2g_ensemble_create", C.c_void_p(fs._fs._ctx_address()),
                  k, nc, n, L, self._ps, float(a_init), nsteps, capi.dptr(av),
                  capi.dptr(ap), 1 if autotune else 0, C.byref(self._e))
        self._bufs = []
        for i, m in enumerate(self.members):
            w, t, d, g = C.c_void_p(), C.c_void_p(), C.c_void_p(), C.c_void_p()
            capi.call("fs2g_ensemble_member", self._e, i, C.byref(w),
                      C.byref(t), C.byref(d), C.byref(g), None, None)
            self._bufs.append((w.value, t.value, d.value, g.value))

    def close(self):
        if self._e:
            capi.lib().fs2g_ensemble_free(self._e)
            self._e = C.c_void_p()
        if self._ps:
            capi.lib().fs2g_power_free(self._ps)
            self._ps = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _view(self, i, which, side):
        import torch
        return torch.as_tensor(_Dev(self._bufs[i][which], (side,) * 3),
                               device="cuda")

    def noise(self, i):
        return self._view(i, 0, self.members[i].nc)

    def target(self, i):
        return self._view(i, 1, self.members[i].n)

    def density(self, i):
        return self._view(i, 2, self.members[i].n)

    def gradient(self, i):
        return self._view(i, 3, self.members[i].nc)

    def set_noise(self, i, w):
        self.noise(i).copy_(w)

    def set_target(self, i, t):
        self.target(i).copy_(t)

    def _sync_torch(self):
        import torch
        torch.cuda.synchronize()

    def forward_member(self, i):
        """Forward only: member i's density buffer (a view)."""
        self._sync_torch()
        capi.call("fs2g_ensemble_forward_member", self._e, i)
        return self.density(i)

    def run(self, graph=True):
        """One forward + loss + backward of every member (asynchronous)."""
        self._sync_torch()
        capi.call("fs2g_ensemble_run", self._e,
                  capi.ENSEMBLE_GRAPH if graph else capi.ENSEMBLE_LOOP)

    def losses(self):
        out = (C.c_double * len(self.members))()
        capi.call("fs2g_ensemble_losses", self._e, out)
        return np.array(out[:], dtype=np.float64)

    def graph_kernels(self):
        """Kernel launches in one graph replay."""
        k = C.c_long()
        capi.call("fs2g_ensemble_graph_kernels", self._e, C.byref(k))
        return k.value

    def tuning(self):
        """[(engine, members per chunk, ms)] chosen for each member's size
        class (ms: the class's forward + loss + backward as tuned)."""
        res = []
        for i in range(len(self.members)):
            e, t, ms = C.c_int(), C.c_int(), C.c_double()
            capi.call("fs2g_ensemble_tuning", self._e, i, C.byref(e),
                      C.byref(t), C.byref(ms))
            res.append(("cufft" if e.value == capi.FFT_CUFFT else "fused",
                        t.value, ms.value))
        return res
