// pm_kernels.cu -- particle-mesh kernels for sm_100a.
//
// Arithmetic follows the reference loop by loop (py/pm.cpp) with explicit
// round-to-nearest intrinsics, so that no product is fused into an add and
// every float/double promotion happens where the reference's C++ puts it.
// Given the same inputs, wrap, the CIC weights, the k-space force and the
// gather are bitwise equal to the reference's serial arithmetic.  Only the
// order of the deposit's additions (atomics) and the FFTs (cuFFT) differ.
//
// Layouts: particle positions are three planes x0[], x1[], x2[]; the real
// mesh is [n][n][ncz] floats, ncz = 2(n/2+1) (py/pm.cpp:242); the spectrum is
// [n][n][n/2+1] float2 (cuFFT's R2C layout, not FFTW-MPI's transposed one).
//
// Batches (a context holding several same-sized realisations, the
// ensemble's size classes): gridDim.y is the member; member m owns
// particles [m np_m, (m+1) np_m) of the set and the m-th of the stacked
// meshes.  With one member (every public context) blockIdx.y = 0.
#include <algorithm>
#include <cub/cub.cuh>
#include "internal.h"
#include <cmath>
#include "cola_math.cuh"
#include "reduce_pair.cuh"

namespace fs2g {
namespace {

constexpr int TPB = 256;

inline unsigned grid_for(size_t n, int tpb = TPB) {
  return (unsigned)((n + tpb - 1)/tpb);
}

// CIC indices and weights along one axis, py/pm.cpp:85-115 and :156-192:
// X = x*dx_inv (Float), i0 = (int)X, w1 = X - i0, w0 = 1 - w1, then
// i0 >= n -> 0, i1 = i0 + 1 wrapped.  A cell index below 0 (a position below
// -1 cell, which the reference's wrap rules out) is flagged and clamped.
struct Cic1 { int i0, i1; float w0, w1; };

__device__ __forceinline__ Cic1 cic1(float x, float dx_inv, int n, bool& bad) {
  Cic1 c;
  const float X = __fmul_rn(x, dx_inv);
  int i0 = __float2int_rz(X);
  c.w1 = __fsub_rn(X, __int2float_rn(i0));
  c.w0 = __fsub_rn(1.0f, c.w1);
  if(i0 >= n) i0 = 0;
  if(i0 < 0) { bad = true; i0 = 0; }
  int i1 = i0 + 1; if(i1 >= n) i1 -= n;
  c.i0 = i0; c.i1 = i1;
  return c;
}

__device__ __forceinline__ float w3(float a, float b, float c, float d) {
  // a*b*c*d evaluated left to right in float, as fac*wx*wy*wz (py/pm.cpp:122)
  return __fmul_rn(__fmul_rn(__fmul_rn(a, b), c), d);
}

__device__ __forceinline__ void flag(int* err, int code, long long detail) {
  if(atomicCAS(err, 0, code) == 0) err[1] = (int) detail;
}

// x[i], folded into [0, L) first when `wrap` (py/util.h:14-24, the fold
// pm_domain_send_positions applies before every deposit); a changed value
// is stored back, as the reference's wrap does
__device__ __forceinline__ float wrap_load(float* __restrict__ x, size_t i,
                                           float L, bool wrap) {
  const float x0 = x[i];
  if(!wrap) return x0;
  float v = x0;
  if(v < 0) v = __fadd_rn(v, L);
  if(v >= L) v = __fsub_rn(v, L);
  if(__float_as_uint(v) != __float_as_uint(x0)) x[i] = v;
  return v;
}

// Thread t -> particle index for the fused gather.  R = 0: the identity.
// R = nc (np = nc^3, nc % 16 == 0, Lagrangian order (ix nc + iy) nc + iz):
// warp w takes a tile of 2 rows (iy) x 16 iz instead of 32 consecutive iz.
// That is a more compact patch of the initial lattice, so once particles
// cluster a warp's mesh loads touch fewer lines, while 16 neighbours along
// z keep the early, uniform steps' loads coalesced.  A bijection on
// [0, np).  Measured at 512^3 / 1024^3, gather + kick + drift summed over
// the 10-step schedule: 32-particle z runs 57 ms; tiles (ix x iy x iz)
// 1x2x16 50.4, 1x4x8 52.0, 2x2x8 53.8, 1x8x4 57.3, 2x4x4 58.2,
// 4x4x2 81.6 ms.  The atomic deposit keeps z runs: its two- and four-wide
// reductions along a row coalesce there, and tiles gained it nothing
// (1x2x16: 39.7 against 39.9 ms over the schedule).
__device__ __forceinline__ size_t tile_particle(size_t t, unsigned R) {
  if(R == 0) return t;
  const size_t w = t >> 5;
  const unsigned lane = (unsigned) t & 31u;
  const size_t per_band = R/16;
  const size_t band = w/per_band, tc = w - band*per_band;
  return (band*2 + (lane >> 4))*(size_t) R + tc*16 + (lane & 15u);
}

// ---------------------------------------------------------------------
// periodic wrap, py/util.h:14-24 (single fold; stores only what changes)
// ---------------------------------------------------------------------
__global__ void k_wrap(float* __restrict__ x0, float* __restrict__ x1,
                       float* __restrict__ x2, size_t np, float boxsize) {
  const size_t i = blockIdx.x*(size_t)blockDim.x + threadIdx.x;
  if(i >= np) return;
  float* xs[3] = {x0, x1, x2};
#pragma unroll
  for(int k = 0; k < 3; k++) {
    const float x = xs[k][i];
    float v = x;
    if(v < 0) v = __fadd_rn(v, boxsize);
    if(v >= boxsize) v = __fsub_rn(v, boxsize);
    if(v != x || __float_as_uint(v) != __float_as_uint(x)) xs[k][i] = v;
  }
}

// ---------------------------------------------------------------------
// clear_density, py/pm.cpp:414-426: -1 for iz < n.  k_clear leaves the row
// padding untouched as the reference does; k_fill writes -1 over the whole
// padded mesh with 16-byte stores (nothing reads the padding of a real
// mesh: the transforms skip it and copies of the mesh drop it).
// ---------------------------------------------------------------------
__global__ void k_fill(float4* __restrict__ m, size_t n4, float value) {
  const float4 v = make_float4(value, value, value, value);
  for(size_t i = blockIdx.x*(size_t)blockDim.x + threadIdx.x; i < n4;
      i += (size_t) gridDim.x*blockDim.x)
    m[i] = v;
}

__global__ void k_clear(float* __restrict__ mesh, int n, size_t rows) {
  const int ncz = 2*(n/2 + 1);
  for(size_t row = blockIdx.x; row < rows; row += gridDim.x) {
    float2* r = reinterpret_cast<float2*>(mesh + row*(size_t)ncz);
    for(int j = threadIdx.x; j < n/2; j += blockDim.x)
      r[j] = make_float2(-1.0f, -1.0f);
    if((n & 1) && threadIdx.x == 0) mesh[row*(size_t)ncz + n - 1] = -1.0f;
  }
}

// ---------------------------------------------------------------------
// CIC deposit with float atomics, py/pm.cpp:57-139.  Warp-aggregated: lanes
// of a warp whose particles share a base cell (common in collapsed regions)
// first add their 8 weights within the warp, and one lane issues the 8
// atomics.  The per-lane weights are the reference's products.
// ---------------------------------------------------------------------
__global__ void __launch_bounds__(TPB)
k_deposit_atomic(float* __restrict__ x0, float* __restrict__ x1,
                 float* __restrict__ x2, size_t np,
                 float* __restrict__ mesh, int n, float dx_inv, float fac,
                 float boxsize, int wrap, int* __restrict__ err) {
  // np: particles per member
  const size_t il = blockIdx.x*(size_t)blockDim.x + threadIdx.x;
  const size_t i = blockIdx.y*np + il;
  const bool active = il < np;
  const int ncz = 2*(n/2 + 1);
  mesh += blockIdx.y*((size_t) n*n*ncz);
  bool bad = false;
  Cic1 cx{0, 0, 0.f, 0.f}, cy{0, 0, 0.f, 0.f}, cz{0, 0, 0.f, 0.f};
  if(active) {
    cx = cic1(wrap_load(x0, i, boxsize, wrap), dx_inv, n, bad);
    cy = cic1(wrap_load(x1, i, boxsize, wrap), dx_inv, n, bad);
    cz = cic1(wrap_load(x2, i, boxsize, wrap), dx_inv, n, bad);
    if(bad) flag(err, DEV_POSITION_OUT_OF_RANGE, (long long) i);
  }
  const bool live = active && !bad;
  float w[8];
  w[0] = w3(fac, cx.w0, cy.w0, cz.w0);
  w[1] = w3(fac, cx.w0, cy.w0, cz.w1);
  w[2] = w3(fac, cx.w0, cy.w1, cz.w0);
  w[3] = w3(fac, cx.w0, cy.w1, cz.w1);
  w[4] = w3(fac, cx.w1, cy.w0, cz.w0);
  w[5] = w3(fac, cx.w1, cy.w0, cz.w1);
  w[6] = w3(fac, cx.w1, cy.w1, cz.w0);
  w[7] = w3(fac, cx.w1, cy.w1, cz.w1);

  // group lanes with the same base cell
  const unsigned live_mask = __ballot_sync(0xffffffffu, live);
  if(!live) return;
  const unsigned key = ((unsigned) cx.i0*(unsigned) n + (unsigned) cy.i0)*
                       (unsigned) n + (unsigned) cz.i0;
  const unsigned peers = __match_any_sync(live_mask, key);
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(peers) - 1;
  if(__popc(peers) > 1) {
    // sum the group's weights into the leader, in ascending lane order
    unsigned rest = peers & ~(1u << leader);
    float acc[8];
#pragma unroll
    for(int o = 0; o < 8; o++) acc[o] = w[o];
    while(rest) {
      const int src = __ffs(rest) - 1;
      rest &= rest - 1;
#pragma unroll
      for(int o = 0; o < 8; o++) {
        const float v = __shfl_sync(peers, w[o], src);
        if(lane == leader) acc[o] = __fadd_rn(acc[o], v);
      }
    }
    if(lane != leader) return;
#pragma unroll
    for(int o = 0; o < 8; o++) w[o] = acc[o];
  }
  const size_t total = (size_t) n*n*ncz;
  const size_t r00 = ((size_t) cx.i0*n + cy.i0)*ncz;
  const size_t r01 = ((size_t) cx.i0*n + cy.i1)*ncz;
  const size_t r10 = ((size_t) cx.i1*n + cy.i0)*ncz;
  const size_t r11 = ((size_t) cx.i1*n + cy.i1)*ncz;
  red_pair(mesh, total, r00, cz.i0, cz.i1, w[0], w[1]);
  red_pair(mesh, total, r01, cz.i0, cz.i1, w[2], w[3]);
  red_pair(mesh, total, r10, cz.i0, cz.i1, w[4], w[5]);
  red_pair(mesh, total, r11, cz.i0, cz.i1, w[6], w[7]);
}

// ---------------------------------------------------------------------
// compute_force_mesh k-space part, py/pm.cpp:468-502, per axis:
// f1 = -1/n^3/(2 pi/L) (Float), k_i = i <= n/2 ? i : i - n (x, y), k_z = iz,
// f2 = f1/(kx^2 + ky^2 + kz^2)*k_axis (Float), fk = (-f2 d_im, f2 d_re),
// fk(0) = 0.
// On the kz = 0 and kz = n/2 planes the result is replaced by its Hermitian
// part (F(k) + conj F(-k))/2.  A C2R that transforms x and y first and keeps
// the real part along z -- FFTW's rdft2 and pocketfft -- computes exactly
// that from a spectrum that is not Hermitian there (the +n/2 Nyquist
// convention makes the axis component anti-Hermitian on its Nyquist line);
// cuFFT is only defined for Hermitian input, so the projection is explicit.
// ---------------------------------------------------------------------
// the three axes' k-space force of one mode: f1/(k^2) is the same Float
// for every axis (the reference's f1/(...)*k[axis] divides first), so it
// is evaluated once and multiplied by each k_axis
__device__ __forceinline__ void force_k3_value(const float2* __restrict__ dk,
                                               int ix, int iy, int iz, int n,
                                               int nckz, float f1,
                                               float2 (&F)[3]) {
  if(ix == 0 && iy == 0 && iz == 0) {
    F[0] = F[1] = F[2] = make_float2(0.0f, 0.0f);
    return;
  }
  const int kx = ix <= n/2 ? ix : ix - n;
  const int ky = iy <= n/2 ? iy : iy - n;
  const float fx = (float) kx, fy = (float) ky, fz = (float) iz;
  const float ksq = __fadd_rn(__fadd_rn(__fmul_rn(fx, fx), __fmul_rn(fy, fy)),
                              __fmul_rn(fz, fz));
  const float q = __fdiv_rn(f1, ksq);
  const float2 d = dk[((size_t) ix*n + iy)*nckz + iz];
  const float ka[3] = {fx, fy, fz};
#pragma unroll
  for(int a = 0; a < 3; a++) {
    const float f2 = __fmul_rn(q, ka[a]);
    F[a] = make_float2(__fmul_rn(-f2, d.y), __fmul_rn(f2, d.x));
  }
}

// All three axes in one pass over delta(k), which is read once instead of
// once per axis.  A flat index over the
// member's n^2 (n/2+1) modes keeps whole blocks busy when n/2+1 is small
// (one row per block left most threads idle at the ensemble's sizes).
__global__ void __launch_bounds__(TPB)
k_force_k3(const float2* __restrict__ dk, float2* __restrict__ f0,
           float2* __restrict__ f1o, float2* __restrict__ f2o, int n,
           float f1) {
  const int nckz = n/2 + 1;
  const size_t mo = blockIdx.y*((size_t) n*n*nckz);      // member
  dk += mo; f0 += mo; f1o += mo; f2o += mo;
  const unsigned total = (unsigned)((size_t) n*n*nckz);
  for(unsigned e = blockIdx.x*blockDim.x + threadIdx.x; e < total;
      e += gridDim.x*blockDim.x) {
    const unsigned row = e/(unsigned) nckz;
    const int iz = (int)(e - row*(unsigned) nckz);
    const int ix = (int)(row/(unsigned) n), iy = (int)(row % (unsigned) n);
    float2 F[3];
    force_k3_value(dk, ix, iy, iz, n, nckz, f1, F);
    if(iz == 0 || iz == n/2) {
      const int mx = ix == 0 ? 0 : n - ix, my = iy == 0 ? 0 : n - iy;
      float2 M[3];
      force_k3_value(dk, mx, my, iz, n, nckz, f1, M);
#pragma unroll
      for(int a = 0; a < 3; a++)
        F[a] = make_float2(__fmul_rn(0.5f, __fadd_rn(F[a].x, M[a].x)),
                           __fmul_rn(0.5f, __fsub_rn(F[a].y, M[a].y)));
    }
    f0[e] = F[0];
    f1o[e] = F[1];
    f2o[e] = F[2];
  }
}

// ---------------------------------------------------------------------
// force_at_particle_locations for all three axes, py/pm.cpp:142-220:
// f = (g000 wx0 wy0 wz0 + g001 wx0 wy0 wz1 + g010 ... + g011 ...)
//   + (the same four terms at ix1 with wx1), each product left to right.
// Positions are read once for the three force meshes.
// ---------------------------------------------------------------------
__device__ __forceinline__ float gather1(const float* __restrict__ g,
                                         size_t r00, size_t r01, size_t r10,
                                         size_t r11, const Cic1& cx,
                                         const Cic1& cy, const Cic1& cz) {
  const float a0 = w3(g[r00 + cz.i0], cx.w0, cy.w0, cz.w0);
  const float a1 = w3(g[r00 + cz.i1], cx.w0, cy.w0, cz.w1);
  const float a2 = w3(g[r01 + cz.i0], cx.w0, cy.w1, cz.w0);
  const float a3 = w3(g[r01 + cz.i1], cx.w0, cy.w1, cz.w1);
  const float b0 = w3(g[r10 + cz.i0], cx.w1, cy.w0, cz.w0);
  const float b1 = w3(g[r10 + cz.i1], cx.w1, cy.w0, cz.w1);
  const float b2 = w3(g[r11 + cz.i0], cx.w1, cy.w1, cz.w0);
  const float b3 = w3(g[r11 + cz.i1], cx.w1, cy.w1, cz.w1);
  const float A = __fadd_rn(__fadd_rn(__fadd_rn(a0, a1), a2), a3);
  const float B = __fadd_rn(__fadd_rn(__fadd_rn(b0, b1), b2), b3);
  return __fadd_rn(__fadd_rn(0.0f, A), B);
}

__global__ void __launch_bounds__(TPB)
k_gather3(const float* __restrict__ x0, const float* __restrict__ x1,
          const float* __restrict__ x2, size_t np,
          const float* __restrict__ gx, const float* __restrict__ gy,
          const float* __restrict__ gz, int n, float dx_inv,
          float* __restrict__ f0, float* __restrict__ f1,
          float* __restrict__ f2, int* __restrict__ err,
          unsigned R) {
  // np: particles per member
  const size_t t = blockIdx.x*(size_t)blockDim.x + threadIdx.x;
  if(t >= np) return;
  const size_t i = blockIdx.y*np + tile_particle(t, R);   // as in k_gather4_kd
  const int ncz = 2*(n/2 + 1);
  const size_t mo = blockIdx.y*((size_t) n*n*ncz);
  gx += mo; gy += mo; gz += mo;
  bool bad = false;
  const Cic1 cx = cic1(x0[i], dx_inv, n, bad);
  const Cic1 cy = cic1(x1[i], dx_inv, n, bad);
  const Cic1 cz = cic1(x2[i], dx_inv, n, bad);
  if(bad) {
    flag(err, DEV_POSITION_OUT_OF_RANGE, (long long) i);
    f0[i] = f1[i] = f2[i] = 0.0f;
    return;
  }
  const size_t r00 = ((size_t) cx.i0*n + cy.i0)*ncz;
  const size_t r01 = ((size_t) cx.i0*n + cy.i1)*ncz;
  const size_t r10 = ((size_t) cx.i1*n + cy.i0)*ncz;
  const size_t r11 = ((size_t) cx.i1*n + cy.i1)*ncz;
  f0[i] = gather1(gx, r00, r01, r10, r11, cx, cy, cz);
  f1[i] = gather1(gy, r00, r01, r10, r11, cx, cy, cz);
  f2[i] = gather1(gz, r00, r01, r10, r11, cx, cy, cz);
}

// The same CIC sums over the fused path's interleaved force mesh
// ((f_x, f_y, f_z, 0) per cell, [n][n][n]): one 16-byte load per corner,
// 8 per particle instead of 24 scalar ones, so that a warp whose particles
// are spread over many mesh rows (clustered, late times) issues a third of
// the L1/L2 requests.  Products and summation order are gather1's.
// (A 12-byte layout -- (f_x, f_y) and f_z in two meshes, an 8-byte and a
// 4-byte load per corner -- saves IZ 4.3 GB of writes and the gather as
// much of reads, but measured slower at 512^3 / 1024^3: IZ 5.52 -> 4.97 ms,
// gather + kick + drift 5.05 -> 6.69 ms per step.)
__device__ __forceinline__ float cic_sum(float v000, float v001, float v010,
                                         float v011, float v100, float v101,
                                         float v110, float v111,
                                         const Cic1& cx, const Cic1& cy,
                                         const Cic1& cz) {
  const float a0 = w3(v000, cx.w0, cy.w0, cz.w0);
  const float a1 = w3(v001, cx.w0, cy.w0, cz.w1);
  const float a2 = w3(v010, cx.w0, cy.w1, cz.w0);
  const float a3 = w3(v011, cx.w0, cy.w1, cz.w1);
  const float b0 = w3(v100, cx.w1, cy.w0, cz.w0);
  const float b1 = w3(v101, cx.w1, cy.w0, cz.w1);
  const float b2 = w3(v110, cx.w1, cy.w1, cz.w0);
  const float b3 = w3(v111, cx.w1, cy.w1, cz.w1);
  const float A = __fadd_rn(__fadd_rn(__fadd_rn(a0, a1), a2), a3);
  const float B = __fadd_rn(__fadd_rn(__fadd_rn(b0, b1), b2), b3);
  return __fadd_rn(__fadd_rn(0.0f, A), B);
}

__global__ void __launch_bounds__(TPB)
k_gather4(const float* __restrict__ x0, const float* __restrict__ x1,
          const float* __restrict__ x2, size_t np,
          const float4* __restrict__ g, int n, float dx_inv,
          float* __restrict__ f0, float* __restrict__ f1,
          float* __restrict__ f2, int* __restrict__ err,
          unsigned R) {
  const size_t t = blockIdx.x*(size_t)blockDim.x + threadIdx.x;
  if(t >= np) return;
  const size_t i = tile_particle(t, R);       // as in k_gather4_kd
  bool bad = false;
  const Cic1 cx = cic1(x0[i], dx_inv, n, bad);
  const Cic1 cy = cic1(x1[i], dx_inv, n, bad);
  const Cic1 cz = cic1(x2[i], dx_inv, n, bad);
  if(bad) {
    flag(err, DEV_POSITION_OUT_OF_RANGE, (long long) i);
    f0[i] = f1[i] = f2[i] = 0.0f;
    return;
  }
  const size_t r00 = ((size_t) cx.i0*n + cy.i0)*n;
  const size_t r01 = ((size_t) cx.i0*n + cy.i1)*n;
  const size_t r10 = ((size_t) cx.i1*n + cy.i0)*n;
  const size_t r11 = ((size_t) cx.i1*n + cy.i1)*n;
  const float4 c000 = __ldg(g + r00 + cz.i0), c001 = __ldg(g + r00 + cz.i1);
  const float4 c010 = __ldg(g + r01 + cz.i0), c011 = __ldg(g + r01 + cz.i1);
  const float4 c100 = __ldg(g + r10 + cz.i0), c101 = __ldg(g + r10 + cz.i1);
  const float4 c110 = __ldg(g + r11 + cz.i0), c111 = __ldg(g + r11 + cz.i1);
  f0[i] = cic_sum(c000.x, c001.x, c010.x, c011.x, c100.x, c101.x, c110.x,
                  c111.x, cx, cy, cz);
  f1[i] = cic_sum(c000.y, c001.y, c010.y, c011.y, c100.y, c101.y, c110.y,
                  c111.y, cx, cy, cz);
  f2[i] = cic_sum(c000.z, c001.z, c010.z, c011.z, c100.z, c101.z, c110.z,
                  c111.z, cx, cy, cz);
}

// The gather over the interleaved force mesh followed, for the same
// particle, by the COLA kick and drift of the step (fs2g_cola_step): f is
// written as k_gather4 writes it, then v and x are updated exactly as
// k_cola4<2> would, but x and f come from registers instead of HBM.
// Planes of the particle set start at base + p*stride (x 0-2, v 3-5, dx1
// 6-8, dx2 9-11, force 12-14).
__global__ void __launch_bounds__(TPB)
k_gather4_kd(float* __restrict__ base, size_t stride, size_t np,
             const float4* __restrict__ g, int n, float dx_inv, KickCoef kc,
             DriftCoef dc, int* __restrict__ err, unsigned R) {
  const size_t t = blockIdx.x*(size_t)blockDim.x + threadIdx.x;
  if(t >= np) return;
  const size_t i = tile_particle(t, R);
  float xr[3], fr[3];
#pragma unroll
  for(int c = 0; c < 3; c++) xr[c] = base[c*stride + i];
  bool bad = false;
  const Cic1 cx = cic1(xr[0], dx_inv, n, bad);
  const Cic1 cy = cic1(xr[1], dx_inv, n, bad);
  const Cic1 cz = cic1(xr[2], dx_inv, n, bad);
  if(bad) {
    flag(err, DEV_POSITION_OUT_OF_RANGE, (long long) i);
    fr[0] = fr[1] = fr[2] = 0.0f;
  }
  else {
    const size_t r00 = ((size_t) cx.i0*n + cy.i0)*n;
    const size_t r01 = ((size_t) cx.i0*n + cy.i1)*n;
    const size_t r10 = ((size_t) cx.i1*n + cy.i0)*n;
    const size_t r11 = ((size_t) cx.i1*n + cy.i1)*n;
    const float4 c000 = __ldg(g + r00 + cz.i0), c001 = __ldg(g + r00 + cz.i1);
    const float4 c010 = __ldg(g + r01 + cz.i0), c011 = __ldg(g + r01 + cz.i1);
    const float4 c100 = __ldg(g + r10 + cz.i0), c101 = __ldg(g + r10 + cz.i1);
    const float4 c110 = __ldg(g + r11 + cz.i0), c111 = __ldg(g + r11 + cz.i1);
    fr[0] = cic_sum(c000.x, c001.x, c010.x, c011.x, c100.x, c101.x, c110.x,
                    c111.x, cx, cy, cz);
    fr[1] = cic_sum(c000.y, c001.y, c010.y, c011.y, c100.y, c101.y, c110.y,
                    c111.y, cx, cy, cz);
    fr[2] = cic_sum(c000.z, c001.z, c010.z, c011.z, c100.z, c101.z, c110.z,
                    c111.z, cx, cy, cz);
  }
#pragma unroll
  for(int c = 0; c < 3; c++) {
    base[(12 + c)*stride + i] = fr[c];
    const float d1 = base[(6 + c)*stride + i], d2 = base[(9 + c)*stride + i];
    const float v = cola_kick1(base[(3 + c)*stride + i], fr[c], d1, d2, kc);
    base[(3 + c)*stride + i] = v;
    base[c*stride + i] = cola_drift1(xr[c], v, d1, d2, dc);
  }
}

// dense[n][n][n] = component `comp` of the interleaved force mesh
__global__ void k_extract(const float4* __restrict__ g, int comp,
                          float* __restrict__ dense, size_t cells) {
  for(size_t i = blockIdx.x*(size_t)blockDim.x + threadIdx.x; i < cells;
      i += (size_t) gridDim.x*blockDim.x)
    dense[i] = reinterpret_cast<const float*>(g + i)[comp];
}

// py/py_fft.cpp:57-85: fx[ix,iy,iz] = (ix*nc + iy)*nc + iz + 1
__global__ void k_fill_test_data(float* __restrict__ fx, int n) {
  const int ncz = 2*(n/2 + 1);
  const size_t row = blockIdx.x;
  for(int iz = threadIdx.x; iz < n; iz += blockDim.x) {
    const size_t g = row*(size_t) n + iz;
    fx[row*ncz + iz] = (float)(g + 1);
  }
}

// sum of the mesh (iz < n) in double, py/pm.cpp:364-370
__global__ void k_density_sum(const float* __restrict__ mesh, int n,
                              size_t rows, double* __restrict__ out) {
  const int ncz = 2*(n/2 + 1);
  double s = 0.0;
  for(size_t row = blockIdx.x; row < rows; row += gridDim.x)
    for(int iz = threadIdx.x; iz < n; iz += blockDim.x)
      s += (double) mesh[row*ncz + iz];
  typedef cub::BlockReduce<double, TPB> BR;
  __shared__ typename BR::TempStorage tmp;
  const double t = BR(tmp).Sum(s);
  if(threadIdx.x == 0) atomicAdd(out, t);
}

}  // namespace

// ---------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------
void launch_wrap(fs2g_ctx* ctx, fs2g_particles* p) {
  if(p->np_local == 0) return;
  k_wrap<<<grid_for(p->np_local), TPB, 0, ctx->stream>>>(
      p->plane(FS2G_FIELD_X, 0), p->plane(FS2G_FIELD_X, 1),
      p->plane(FS2G_FIELD_X, 2), p->np_local, (float) p->boxsize);
  FS2G_LAUNCHED(ctx);
}

void launch_clear_density(fs2g_ctx* ctx, float* mesh, int n) {
  // every member's mesh: the stacked meshes are contiguous
  const size_t total = (size_t) n*n*(2*(n/2 + 1))*ctx->batch;
  if(total % 4 == 0) {
    const size_t n4 = total/4;
    const unsigned blocks = (unsigned) std::min<size_t>((n4 + TPB - 1)/TPB,
                                                        (size_t) ctx->sm_count*32);
    k_fill<<<blocks, TPB, 0, ctx->stream>>>(reinterpret_cast<float4*>(mesh), n4, -1.0f);
  }
  else {
    const size_t rows = (size_t) n*n*ctx->batch;
    const unsigned blocks = (unsigned) std::min<size_t>(rows, (size_t) ctx->sm_count*16);
    k_clear<<<blocks, TPB, 0, ctx->stream>>>(mesh, n, rows);
  }
  FS2G_LAUNCHED(ctx);
}

// R for tile_particle: nc when np is a cube nc^3 with nc % 16 == 0 (the
// 2LPT lattice); otherwise 0, the identity
static unsigned lattice_side(size_t np) {
  const size_t nc = (size_t) std::llround(std::cbrt((double) np));
  return (nc > 0 && nc*nc*nc == np && nc % 16 == 0 && nc < (1u << 31)) ? (unsigned) nc : 0u;
}

void launch_deposit_atomic(fs2g_ctx* ctx, fs2g_particles* p, float* mesh,
                           int n, float boxsize, float fac, bool wrap) {
  if(p->np_local == 0) return;
  const float dx_inv = (float) n / boxsize;          // py/pm.cpp:77
  const size_t npm = member_np(ctx, p);
  k_deposit_atomic<<<dim3(grid_for(npm), ctx->batch), TPB, 0, ctx->stream>>>(
      p->plane(FS2G_FIELD_X, 0), p->plane(FS2G_FIELD_X, 1),
      p->plane(FS2G_FIELD_X, 2), npm, mesh, n, dx_inv, fac,
      (float) p->boxsize, wrap ? 1 : 0, ctx->d_err);
  FS2G_LAUNCHED(ctx);
}

void launch_force_k3(fs2g_ctx* ctx, const float2* delta_k, float2* const fk[3],
                     int n, float f1) {
  const size_t total = (size_t) n*n*(n/2 + 1);
  const unsigned blocks = (unsigned) std::min<size_t>(
      (total + TPB - 1)/TPB, (size_t) ctx->sm_count*16);
  k_force_k3<<<dim3(blocks, ctx->batch), TPB, 0, ctx->stream>>>(
      delta_k, fk[0], fk[1], fk[2], n, f1);
  FS2G_LAUNCHED(ctx);
}

void launch_gather3(fs2g_ctx* ctx, fs2g_particles* p, const float* fx,
                    const float* fy, const float* fz, int n, float boxsize) {
  if(p->np_local == 0) return;
  const float dx_inv = (float) n / boxsize;          // py/pm.cpp:146
  const size_t npm = member_np(ctx, p);
  k_gather3<<<dim3(grid_for(npm), ctx->batch), TPB, 0, ctx->stream>>>(
      p->plane(FS2G_FIELD_X, 0), p->plane(FS2G_FIELD_X, 1),
      p->plane(FS2G_FIELD_X, 2), npm, fx, fy, fz, n, dx_inv,
      p->plane(FS2G_FIELD_FORCE, 0), p->plane(FS2G_FIELD_FORCE, 1),
      p->plane(FS2G_FIELD_FORCE, 2), ctx->d_err, lattice_side(npm));
  FS2G_LAUNCHED(ctx);
}

void launch_gather4(fs2g_ctx* ctx, fs2g_particles* p, const float4* f4, int n,
                    float boxsize) {
  if(p->np_local == 0) return;
  const float dx_inv = (float) n / boxsize;
  k_gather4<<<grid_for(p->np_local), TPB, 0, ctx->stream>>>(
      p->plane(FS2G_FIELD_X, 0), p->plane(FS2G_FIELD_X, 1),
      p->plane(FS2G_FIELD_X, 2), p->np_local, f4, n, dx_inv,
      p->plane(FS2G_FIELD_FORCE, 0), p->plane(FS2G_FIELD_FORCE, 1),
      p->plane(FS2G_FIELD_FORCE, 2), ctx->d_err, lattice_side(p->np_local));
  FS2G_LAUNCHED(ctx);
}

void launch_gather4_kick_drift(fs2g_ctx* ctx, fs2g_particles* p,
                               const float4* f4, int n, float boxsize,
                               KickCoef k, DriftCoef d) {
  if(p->np_local == 0) return;
  const float dx_inv = (float) n / boxsize;
  k_gather4_kd<<<grid_for(p->np_local), TPB, 0, ctx->stream>>>(
      p->d_planes, p->stride, p->np_local, f4, n, dx_inv, k, d, ctx->d_err,
      lattice_side(p->np_local));
  FS2G_LAUNCHED(ctx);
}

void launch_extract_component(fs2g_ctx* ctx, const float4* f4, int comp,
                              float* dense, int n) {
  const size_t cells = (size_t) n*n*n;
  const unsigned blocks = (unsigned) std::min<size_t>((cells + TPB - 1)/TPB,
                                                      (size_t) ctx->sm_count*32);
  k_extract<<<blocks, TPB, 0, ctx->stream>>>(f4, comp, dense, cells);
  FS2G_LAUNCHED(ctx);
}

void launch_fill_test_data(fs2g_ctx* ctx, float* fx, int n) {
  k_fill_test_data<<<(unsigned)((size_t) n*n), 128, 0, ctx->stream>>>(fx, n);
  FS2G_LAUNCHED(ctx);
}

void launch_density_sum(fs2g_ctx* ctx, const float* mesh, int n,
                        double* d_sum) {
  const size_t rows = (size_t) n*n;
  const unsigned blocks = (unsigned) std::min<size_t>(rows, (size_t) ctx->sm_count*8);
  FS2G_CUDA(cudaMemsetAsync(d_sum, 0, sizeof(double), ctx->stream));
  k_density_sum<<<blocks, TPB, 0, ctx->stream>>>(mesh, n, rows, d_sum);
  FS2G_LAUNCHED(ctx);
}

}  // namespace fs2g
