// cola_math.cuh -- the per-component COLA kick and drift of one particle,
// with the reference's promotions (py/cola.cpp:79-88, :117-124):
//   kick:  a = (Float)((-1.5*om) * (double)(f + dx1*q1 + dx2*q2));
//          v = v + a*kick_factor                       (all else float)
//   drift: x = (Float)((double)x + ((double)v*dt + (double)(dx1*da1 + dx2*da2)))
// Shared by the COLA streams and the gather that applies them in its
// epilogue.  Device code only.
#pragma once
#include "internal.h"

namespace fs2g {

__device__ __forceinline__ float cola_kick1(float v, float f, float d1,
                                            float d2, const KickCoef& k) {
  const float s = __fadd_rn(__fadd_rn(f, __fmul_rn(d1, k.q1)),
                            __fmul_rn(d2, k.q2));
  const float a = __double2float_rn(__dmul_rn(k.neg15om, (double) s));
  return __fadd_rn(v, __fmul_rn(a, k.kick_factor));
}

__device__ __forceinline__ float cola_drift1(float x, float v, float d1,
                                             float d2, const DriftCoef& d) {
  const double vt = __dmul_rn((double) v, d.dt);
  const float b = __fadd_rn(__fmul_rn(d1, d.da1), __fmul_rn(d2, d.da2));
  const double r = __dadd_rn(vt, (double) b);
  return __double2float_rn(__dadd_rn((double) x, r));
}

}  // namespace fs2g
