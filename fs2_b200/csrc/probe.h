// probe.h -- profiling and test entry points of libfs2gpu that are not
// part of the public C ABI (include/fs2gpu.h).  Exported from the library
// for the test suite and profiler captures only; no reference counterpart.
#pragma once

#ifdef __cplusplus
extern "C" {
#endif

/* Runs one pass of the 1024^3 fused Poisson pipeline (0 FZ, 1 FY, 2 XX, 3 IY, 4 IZ) `reps`
   times on the current device.  The pass covers a slab of `planes` x
   planes (XX: 32 or 64 ky rows, so planes must be 32 or 64) of seeded data.  The slab
   keeps the buffers to about 1.2 GB at 32 planes, small enough for a
   full profiler capture, whereas the whole pipeline holds about 40 GB.
   It allocates and frees its own buffers, needs no context, and returns
   the average launch time in *ms.  The results are discarded. */
int fs2g_fused_pass_probe(int pass, int planes, int reps, double* ms);

#ifdef __cplusplus
}
#endif
