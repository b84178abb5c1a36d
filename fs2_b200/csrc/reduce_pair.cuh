// reduce_pair.cuh -- two float reductions into neighbouring mesh cells as
// one vector reduction where their alignment allows.  Device code only;
// shared by the CIC deposit (pm_kernels.cu) and its transpose in the
// adjoint (adjoint_kernels.cu).
#pragma once
#include <cstdint>
#include <cstddef>

namespace fs2g {

// mesh[r + z0] += a and mesh[r + z1] += b.  When the two cells are
// neighbours, one vector reduction replaces two: a two-wide one when they
// are an aligned 8-byte pair (half the cases), a four-wide one with +0 in
// the two outer lanes when they sit in the middle of an aligned 16-byte
// chunk (a quarter).  Adding +0 leaves a cell bit for bit unchanged (no
// cell holds -0: the mesh starts at -1 and receives non-negative weights;
// in the adjoint's zeroed meshes a -0 cell may become +0, the same number).
// Chunks stay inside the mesh's `total` floats.
static __device__ __forceinline__ void red_pair(float* __restrict__ mesh,
                                                size_t total, size_t r, int z0,
                                                int z1, float a, float b) {
  const size_t i0 = r + z0;
  const int o = (int)((reinterpret_cast<uintptr_t>(mesh + i0) >> 2) & 3);
  if(z1 == z0 + 1 && (o & 1) == 0) {
    // an aligned pair of floats: one two-wide reduction, no extra lanes
    asm volatile("red.global.v2.f32.add [%0], {%1, %2};"
                 :: "l"(mesh + i0), "f"(a), "f"(b) : "memory");
  }
  else if(z1 == z0 + 1 && o == 1 && i0 - 1 + 4 <= total) {
    asm volatile("red.global.v4.f32.add [%0], {%1, %2, %3, %4};"
                 :: "l"(mesh + i0 - 1), "f"(0.0f), "f"(a), "f"(b), "f"(0.0f)
                 : "memory");
  }
  else {
    atomicAdd(mesh + i0, a);
    atomicAdd(mesh + r + z1, b);
  }
}

}  // namespace fs2g
