"""The allocation-free CIC density, fs2g_cic_density_noalloc.

Callers that own all device memory themselves, or that call from a time loop
that cannot absorb cudaFree's device-wide synchronisation, cannot let the
library allocate.  This entry point keeps its scratch in a fixed file-scope
device array instead.  The test calls it through the C ABI twice in a row on
different particle sets (the second call reuses the array the first one
left behind) and checks each result bit for bit against the allocating
entry point, fs2g_pm_compute_density in deterministic mode (the same
kernels), and against the oracle with the density tolerance of the other
parity tests.  It also checks that the second call leaves the device's free
memory unchanged.  The file sorts last so that a failure here stops a -x run
only after every other test has run.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _positions(n_side, boxsize, seed):
    rng = np.random.default_rng(seed)
    g = (np.stack(np.meshgrid(*[np.arange(n_side)] * 3, indexing="ij"), -1)
         .reshape(-1, 3) + 0.5) * (boxsize / n_side)
    x = g + rng.normal(0, 0.6 * boxsize / n_side, g.shape)
    clump = rng.normal(0.4 * boxsize, 0.02 * boxsize, (len(x) // 8, 3))
    x[: len(clump)] = clump
    return np.mod(x, boxsize).astype(np.float32)


def test_noalloc_density_matches_allocating_entry_point(oracle_mod):
    import torch
    import fs2_b200.fs as fs
    from fs2_b200 import capi

    L = capi.lib()
    n, box, pm_factor = 64, 64.0, 2.0
    ncz = 2 * (n // 2 + 1)
    fs.pm.init(n, pm_factor, box)
    fs.pm.set_deposit_mode("deterministic")
    try:
        for call, (seed, side) in enumerate(((21, 32), (22, 24))):
            x = _positions(side, box, seed)
            np_ = len(x)
            assert np_ <= 262144
            p = fs.Particles(np_, box)
            p.set("x", x)
            want = fs.pm.compute_density(p).asarray().copy()

            base, stride = C.c_void_p(), C.c_size_t()
            pa = C.c_void_p(fs._fs._particles_address(p._particles))
            capi.call("fs2g_particles_device_field", pa, capi.FIELD_X,
                      C.byref(base), C.byref(stride))
            fs._fs._synchronize()
            plane = stride.value * 4
            out = torch.full((n * n * ncz,), 7.0, dtype=torch.float32,
                             device="cuda")
            torch.cuda.synchronize()
            free0 = torch.cuda.mem_get_info()[0]
            rc = L.fs2g_cic_density_noalloc(
                C.c_void_p(base.value), C.c_void_p(base.value + plane),
                C.c_void_p(base.value + 2 * plane), np_,
                C.c_void_p(out.data_ptr()), n, box, pm_factor, None)
            assert rc == 0, capi.last_error()
            free1 = torch.cuda.mem_get_info()[0]
            if call == 1:
                # the first call may load the module (and its scratch array);
                # after that, a call allocates nothing on the device
                assert free1 == free0
            mesh = out.view(n, n, ncz).cpu().numpy()
            got = mesh[:, :, :n]
            assert np.array_equal(got, want)
            pm = oracle_mod.PM(n, pm_factor, box)
            d_or = oracle_mod.unpad(pm.density(x))
            err = np.linalg.norm((got - d_or).astype(np.float64)) / \
                np.linalg.norm(d_or.astype(np.float64))
            assert err <= 1e-5, err
            assert np.abs(got - d_or).max() <= \
                500 * np.finfo(np.float32).eps * max(1.0, np.abs(d_or).max())
            # the padding of the rows is not written
            assert np.all(mesh[:, :, n:] == 7.0)
    finally:
        fs.pm.set_deposit_mode("atomic")


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    from fs2_b200 import capi
    L = capi.lib()
    # small real device buffers: if the checks ever let a call through, the
    # kernels write inside these instead of at an invalid address
    n = 64
    mesh = torch.zeros(n * n * (n + 2), dtype=torch.float32, device="cuda")
    xs = [torch.zeros(1, dtype=torch.float32, device="cuda") for _ in range(3)]
    ptrs = [C.c_void_p(t.data_ptr()) for t in xs]
    big = 262144 + 1
    rc = L.fs2g_cic_density_noalloc(*ptrs, big, C.c_void_p(mesh.data_ptr()),
                                    n, 64.0, 1.0, None)
    assert rc == -5
    assert "FS2G_NOALLOC_MAX_PARTICLES" in capi.last_error()
    rc = L.fs2g_cic_density_noalloc(*ptrs, 1, C.c_void_p(mesh.data_ptr()),
                                    2048, 64.0, 1.0, None)
    assert rc == -5
    assert "FS2G_NOALLOC_MAX_MESH" in capi.last_error()
    torch.cuda.synchronize()
