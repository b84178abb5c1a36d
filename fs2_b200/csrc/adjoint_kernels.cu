// adjoint_kernels.cu -- reverse-mode (adjoint) kernels of the differentiable
// COLA simulation: white noise -> 2LPT -> COLA steps -> CIC density.
//
// No reference counterpart: fs2 has no gradients.  Each kernel here is the
// transpose of one forward operation of this library:
//   k_scatter3        transpose of the 3-component CIC gather (f -> mesh)
//   k_deriv_gather    d/dx of the CIC weights in deposit and gather
//   k_poisson_adj_k   transpose of the spectral force: -sum_a M_a G_a
//   k_cola_adj        transpose of kick then drift
//   k_lpt_* (adj)     transposes of the 2LPT maps from white noise
// A spectral operator C2R(Q R2C(y)) is real-linear; its transpose is
// C2R(conj(Q) R2C(ybar)) with the same C2R, whose real part on the kz = 0 and
// kz = n/2 planes (explicit Hermitian part before cuFFT) makes it exact.
//
// Batched contexts (an ensemble's size class): gridDim.y is the member, as
// in pm_kernels.cu; member m owns particles [m np_m, (m+1) np_m) and the
// m-th of each set of stacked meshes.
#include <algorithm>
#include "internal.h"
#include "reduce_pair.cuh"

namespace fs2g {
namespace {

constexpr int TPB = 256;

inline unsigned grid_for(size_t n, int tpb = TPB) {
  return (unsigned)((n + tpb - 1)/tpb);
}

struct Cic {
  int i0, i1; float w0, w1;
};

__device__ __forceinline__ Cic cic(float x, float dx_inv, int n) {
  Cic c;
  const float X = x*dx_inv;
  int i0 = __float2int_rz(X);
  c.w1 = X - (float) i0;
  c.w0 = 1.0f - c.w1;
  if(i0 >= n) i0 = 0;
  if(i0 < 0) i0 = 0;
  int i1 = i0 + 1; if(i1 >= n) i1 -= n;
  c.i0 = i0; c.i1 = i1;
  return c;
}

// ghat_a[c] += sum_p W(x_p - c) fbar_{p,a}, three meshes
__global__ void __launch_bounds__(TPB)
k_scatter3(const float* __restrict__ x0, const float* __restrict__ x1,
           const float* __restrict__ x2, const float* __restrict__ f0,
           const float* __restrict__ f1, const float* __restrict__ f2,
           size_t np, int n, float dx_inv, float* __restrict__ g0,
           float* __restrict__ g1, float* __restrict__ g2) {
  // np: particles per member
  const size_t il = blockIdx.x*(size_t)blockDim.x + threadIdx.x;
  if(il >= np) return;
  const size_t i = blockIdx.y*np + il;
  const int ncz = 2*(n/2 + 1);
  const size_t mo = blockIdx.y*((size_t) n*n*ncz);
  g0 += mo; g1 += mo; g2 += mo;
  const Cic cx = cic(x0[i], dx_inv, n), cy = cic(x1[i], dx_inv, n),
            cz = cic(x2[i], dx_inv, n);
  const float fa[3] = {f0[i], f1[i], f2[i]};
  float* g[3] = {g0, g1, g2};
  const size_t total = (size_t) n*n*ncz;
  // per (x, y) corner: its two z cells as one reduction where aligned
#pragma unroll
  for(int q = 0; q < 4; q++) {
    const int ix = (q & 2) ? cx.i1 : cx.i0, iy = (q & 1) ? cy.i1 : cy.i0;
    const float wxy = ((q & 2) ? cx.w1 : cx.w0)*((q & 1) ? cy.w1 : cy.w0);
    const float w0 = wxy*cz.w0, w1 = wxy*cz.w1;
    const size_t r = ((size_t) ix*n + iy)*ncz;
#pragma unroll
    for(int a = 0; a < 3; a++)
      red_pair(g[a], total, r, cz.i0, cz.i1, w0*fa[a], w1*fa[a]);
  }
}

// xbar_{p,d} += sum_c dW_c/dx_d [ sum_a fbar_{p,a} g_a[c] + dfac dbar[c] ]
// (g or dbar may be null).  The force meshes g_a are either three padded
// real meshes g0..g2 or, when g4 is given, the fused path's interleaved
// mesh ((f_x, f_y, f_z, 0) per cell, [n][n][n]).
__global__ void __launch_bounds__(TPB)
k_deriv_gather(const float* __restrict__ x0, const float* __restrict__ x1,
               const float* __restrict__ x2, const float* __restrict__ fb0,
               const float* __restrict__ fb1, const float* __restrict__ fb2,
               const float* __restrict__ g0, const float* __restrict__ g1,
               const float* __restrict__ g2, const float4* __restrict__ g4,
               const float* __restrict__ dbar,
               float dfac, size_t np, int n, float dx_inv,
               float* __restrict__ xb0, float* __restrict__ xb1,
               float* __restrict__ xb2) {
  // np: particles per member (the fused mesh g4: one member only)
  const size_t il = blockIdx.x*(size_t)blockDim.x + threadIdx.x;
  if(il >= np) return;
  const size_t i = blockIdx.y*np + il;
  const int ncz = 2*(n/2 + 1);
  const size_t mo = blockIdx.y*((size_t) n*n*ncz);
  if(g0) { g0 += mo; g1 += mo; g2 += mo; }
  if(dbar) dbar += mo;
  const Cic cx = cic(x0[i], dx_inv, n), cy = cic(x1[i], dx_inv, n),
            cz = cic(x2[i], dx_inv, n);
  float fa[3] = {0.f, 0.f, 0.f};
  const bool have_g = g0 || g4;
  if(have_g) { fa[0] = fb0[i]; fa[1] = fb1[i]; fa[2] = fb2[i]; }
  float gx = 0.f, gy = 0.f, gz = 0.f;
#pragma unroll
  for(int o = 0; o < 8; o++) {
    const bool bx = o & 4, by = o & 2, bz = o & 1;
    const size_t row = (size_t)(bx ? cx.i1 : cx.i0)*n + (by ? cy.i1 : cy.i0);
    const int iz = bz ? cz.i1 : cz.i0;
    const size_t idx = row*ncz + iz;
    float s = 0.f;
    if(g4) {
      const float4 v = g4[row*n + iz];
      s = fa[0]*v.x + fa[1]*v.y + fa[2]*v.z;
    }
    else if(g0) s = fa[0]*g0[idx] + fa[1]*g1[idx] + fa[2]*g2[idx];
    if(dbar) s += dfac*dbar[idx];
    const float wx = bx ? cx.w1 : cx.w0, wy = by ? cy.w1 : cy.w0,
                wz = bz ? cz.w1 : cz.w0;
    const float sx = bx ? dx_inv : -dx_inv, sy = by ? dx_inv : -dx_inv,
                sz = bz ? dx_inv : -dx_inv;
    gx += sx*wy*wz*s;
    gy += wx*sy*wz*s;
    gz += wx*wy*sz*s;
  }
  xb0[i] += gx; xb1[i] += gy; xb2[i] += gz;
}

// out(k) = -sum_a M_a(k) G_a(k), M_a = i f1 k_a / k^2 (the force's k
// convention, py/pm.cpp:483-497), Hermitian part on kz = 0 and kz = n/2
__device__ __forceinline__ float2 padj_value(const float2* __restrict__ G0,
                                             const float2* __restrict__ G1,
                                             const float2* __restrict__ G2,
                                             int ix, int iy, int iz, int n,
                                             float f1) {
  if(ix == 0 && iy == 0 && iz == 0) return make_float2(0.f, 0.f);
  const int nckz = n/2 + 1;
  const float kx = (float)(ix <= n/2 ? ix : ix - n);
  const float ky = (float)(iy <= n/2 ? iy : iy - n);
  const float kz = (float) iz;
  const float g = f1/(kx*kx + ky*ky + kz*kz);
  const size_t idx = ((size_t) ix*n + iy)*nckz + iz;
  const float2 a = G0[idx], b = G1[idx], c = G2[idx];
  // s = sum_a k_a G_a ; out = -i g s
  const float sr = kx*a.x + ky*b.x + kz*c.x, si = kx*a.y + ky*b.y + kz*c.y;
  return make_float2(g*si, -g*sr);
}

__global__ void __launch_bounds__(TPB)
k_poisson_adj_k(const float2* __restrict__ G0, const float2* __restrict__ G1,
                const float2* __restrict__ G2, float2* __restrict__ out, int n,
                float f1) {
  // a flat index over the member's modes (a row per block left most
  // threads idle at small n)
  const int nckz = n/2 + 1;
  const size_t mo = blockIdx.y*((size_t) n*n*nckz);     // member
  G0 += mo; G1 += mo; G2 += mo; out += mo;
  const unsigned total = (unsigned)((size_t) n*n*nckz);
  for(unsigned e = blockIdx.x*blockDim.x + threadIdx.x; e < total;
      e += gridDim.x*blockDim.x) {
    const unsigned row = e/(unsigned) nckz;
    const int iz = (int)(e - row*(unsigned) nckz);
    const int ix = (int)(row/(unsigned) n), iy = (int)(row % (unsigned) n);
    float2 v = padj_value(G0, G1, G2, ix, iy, iz, n, f1);
    if(iz == 0 || iz == n/2) {
      const float2 m = padj_value(G0, G1, G2, ix == 0 ? 0 : n - ix,
                                  iy == 0 ? 0 : n - iy, iz, n, f1);
      v = make_float2(0.5f*(v.x + m.x), 0.5f*(v.y - m.y));
    }
    out[e] = v;
  }
}

// transpose of  v' = v + K (f + q1 dx1 + q2 dx2);  x' = x + dt v' + da1 dx1 + da2 dx2
__global__ void __launch_bounds__(TPB)
k_cola_adj(const float* __restrict__ xb, float* __restrict__ vb,
           float* __restrict__ d1b, float* __restrict__ d2b,
           float* __restrict__ fb, size_t np, float K, float q1, float q2,
           float dt, float da1, float da2) {
  const size_t i = blockIdx.x*(size_t)blockDim.x + threadIdx.x;
  if(i >= np) return;
  const float x = xb[i];
  const float v = vb[i] + dt*x;
  d1b[i] += da1*x + K*q1*v;
  d2b[i] += da2*x + K*q2*v;
  fb[i] = K*v;
  vb[i] = v;
}

// ---------------------------------------------------------------------
// 2LPT from white noise
// ---------------------------------------------------------------------
__device__ double spline_logP_d(const SplineDev& s, double lk) {
  int lo = 0, hi = s.n - 1;
  if(lk <= s.knots[0]) lo = 0;
  else if(lk >= s.knots[hi]) lo = hi - 1;
  else {
    while(hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if(s.knots[mid] > lk) hi = mid; else lo = mid;
    }
  }
  const int m = s.n - 1;
  const double t = lk - s.knots[lo];
  return s.coef[lo] + t*(s.coef[m + lo] + t*(s.coef[2*m + lo] + t*s.coef[3*m + lo]));
}

__device__ __forceinline__ double lpt_kv_d(int i, int nc, double dk) {
  return i < nc/2 ? dk*i : -dk*(nc - i);
}

// T(k) = sqrt(P(k) / (V nc^3)), zero at k = 0 and on the Nyquist planes
__device__ __forceinline__ float transfer(const SplineDev& ps, int ix, int iy,
                                          int iz, int nc, double boxsize) {
  if(ix == nc/2 || iy == nc/2 || iz == nc/2) return 0.f;
  if(ix == 0 && iy == 0 && iz == 0) return 0.f;
  const double dk = 2.0*M_PI/boxsize;
  const double kx = lpt_kv_d(ix, nc, dk), ky = lpt_kv_d(iy, nc, dk),
               kz = lpt_kv_d(iz, nc, dk);
  const double k = sqrt(kx*kx + ky*ky + kz*kz);
  const double P = exp(spline_logP_d(ps, log(k)));
  const double V = boxsize*boxsize*boxsize;
  return (float) sqrt(P/(V*(double) nc*nc*nc));
}

// delta(k) = T(k) X(k), in place
__global__ void k_white_to_delta(float2* __restrict__ X, int nc,
                                 double boxsize, SplineDev ps) {
  const int nckz = nc/2 + 1;
  X += blockIdx.y*((size_t) nc*nc*nckz);               // member
  const size_t row = blockIdx.x;
  const int ix = (int)(row / nc), iy = (int)(row % nc);
  for(int iz = threadIdx.x; iz < nckz; iz += blockDim.x) {
    const float t = transfer(ps, ix, iy, iz, nc, boxsize);
    const float2 v = X[row*nckz + iz];
    X[row*nckz + iz] = make_float2(t*v.x, t*v.y);
  }
}

// particle-ordered adjoints -> grid meshes:
//   psibar_i = D1 xbar_i + dx1bar_i,  psi2bar_i = (D2 xbar_i + dx2bar_i)/nc^3
__global__ void k_lpt_adj_to_mesh(const float* __restrict__ xb,
                                  const float* __restrict__ d1b,
                                  const float* __restrict__ d2b, size_t stride,
                                  int nc, float D1, float D2, float inv3,
                                  float* __restrict__ p0, float* __restrict__ p1,
                                  float* __restrict__ p2, float* __restrict__ q0,
                                  float* __restrict__ q1, float* __restrict__ q2) {
  const size_t ip = blockIdx.x*(size_t)blockDim.x + threadIdx.x;
  const size_t np = (size_t) nc*nc*nc;
  if(ip >= np) return;
  const int nczr = 2*(nc/2 + 1);
  // member blockIdx.y: particles from blockIdx.y np, meshes stacked
  xb += blockIdx.y*np; d1b += blockIdx.y*np; d2b += blockIdx.y*np;
  const size_t mo = blockIdx.y*((size_t) nc*nc*nczr);
  p0 += mo; p1 += mo; p2 += mo; q0 += mo; q1 += mo; q2 += mo;
  const size_t iz = ip % nc, t = ip / nc, iy = t % nc, ix = t / nc;
  const size_t idx = (ix*nc + iy)*nczr + iz;
  float* P[3] = {p0, p1, p2};
  float* Q[3] = {q0, q1, q2};
#pragma unroll
  for(int k = 0; k < 3; k++) {
    const float x = xb[k*stride + ip];
    P[k][idx] = D1*x + d1b[k*stride + ip];
    Q[k][idx] = (D2*x + d2b[k*stride + ip])*inv3;
  }
}

// Sbar(k) = sum_i conj(Q_i) Psi2bar_i(k), Q_i = -i k_i/k^2 (2LPT convention,
// py/lpt.cpp:558-583), Hermitian part on kz = 0 and kz = nc/2
__device__ __forceinline__ float2 sbar_value(const float2* const* Pb, int ix,
                                             int iy, int iz, int nc, double dk) {
  if(ix == 0 && iy == 0 && iz == 0) return make_float2(0.f, 0.f);
  const double k[3] = {lpt_kv_d(ix, nc, dk), lpt_kv_d(iy, nc, dk),
                       lpt_kv_d(iz, nc, dk)};
  const double k2 = k[0]*k[0] + k[1]*k[1] + k[2]*k[2];
  const size_t idx = ((size_t) ix*nc + iy)*(nc/2 + 1) + iz;
  double sr = 0, si = 0;
  for(int i = 0; i < 3; i++) {
    const float2 v = Pb[i][idx];
    // conj(-i k_i/k2) = +i k_i/k2
    sr += -(k[i]/k2)*v.y;
    si += (k[i]/k2)*v.x;
  }
  return make_float2((float) sr, (float) si);
}

struct CPtr3 { const float2* p[3]; };
struct CPtr9 { const float2* p[9]; };

__global__ void k_lpt_adj_s(CPtr3 pb, float2* __restrict__ out, int nc,
                            double boxsize) {
  const int nckz = nc/2 + 1;
  const size_t mo = blockIdx.y*((size_t) nc*nc*nckz);   // member
  for(int i = 0; i < 3; i++) pb.p[i] += mo;
  out += mo;
  const size_t row = blockIdx.x;
  const int ix = (int)(row / nc), iy = (int)(row % nc);
  const double dk = 2.0*M_PI/boxsize;
  for(int iz = threadIdx.x; iz < nckz; iz += blockDim.x) {
    float2 v = sbar_value(pb.p, ix, iy, iz, nc, dk);
    if(iz == 0 || iz == nc/2) {
      const float2 m = sbar_value(pb.p, ix == 0 ? 0 : nc - ix,
                                  iy == 0 ? 0 : nc - iy, iz, nc, dk);
      v = make_float2(0.5f*(v.x + m.x), 0.5f*(v.y - m.y));
    }
    out[row*nckz + iz] = v;
  }
}

// psibar_ij = Sbar dS/dpsi_ij in place over the six psi_ij meshes:
// S = p11 (p22 + p33) + p22 p33 - p12^2 - p13^2 - p23^2, order 11 12 13 22 23 33
__global__ void k_lpt_adj_source(int nc, float* __restrict__ a,
                                 float* __restrict__ b, float* __restrict__ c,
                                 float* __restrict__ d, float* __restrict__ e,
                                 float* __restrict__ f,
                                 const float* __restrict__ sbar) {
  const int nczr = 2*(nc/2 + 1);
  const size_t row = blockIdx.x;
  for(int iz = threadIdx.x; iz < nc; iz += blockDim.x) {
    const size_t i = row*nczr + iz;
    const float s = sbar[i];
    const float p11 = a[i], p12 = b[i], p13 = c[i], p22 = d[i], p23 = e[i],
                p33 = f[i];
    a[i] = s*(p22 + p33);
    d[i] = s*(p11 + p33);
    f[i] = s*(p11 + p22);
    b[i] = -2.f*s*p12;
    c[i] = -2.f*s*p13;
    e[i] = -2.f*s*p23;
  }
}

// Wbar(k) = T(k) [ sum_i conj(A_i) Psibar_i + sum_ij B_ij Psibar_ij ],
// A_i = i k_i/k^2, B_ij = -k_i k_j/k^2; Hermitian part on kz = 0, nc/2
__device__ __forceinline__ float2 wbar_value(const float2* const* P, int ix,
                                             int iy, int iz, int nc,
                                             double boxsize,
                                             const SplineDev& ps) {
  const float t = transfer(ps, ix, iy, iz, nc, boxsize);
  if(t == 0.f) return make_float2(0.f, 0.f);
  const double dk = 2.0*M_PI/boxsize;
  const double k[3] = {lpt_kv_d(ix, nc, dk), lpt_kv_d(iy, nc, dk),
                       lpt_kv_d(iz, nc, dk)};
  const double k2 = k[0]*k[0] + k[1]*k[1] + k[2]*k[2];
  const size_t idx = ((size_t) ix*nc + iy)*(nc/2 + 1) + iz;
  double sr = 0, si = 0;
  for(int i = 0; i < 3; i++) {
    const float2 v = P[i][idx];
    // conj(i k_i/k2) v = -i (k_i/k2) v
    sr += (k[i]/k2)*v.y;
    si += -(k[i]/k2)*v.x;
  }
  const int ci[6] = {0, 0, 0, 1, 1, 2}, cj[6] = {0, 1, 2, 1, 2, 2};
  for(int m = 0; m < 6; m++) {
    const float2 v = P[3 + m][idx];
    const double bij = -k[ci[m]]*k[cj[m]]/k2;
    sr += bij*v.x;
    si += bij*v.y;
  }
  return make_float2((float)(t*sr), (float)(t*si));
}

__global__ void k_lpt_adj_w(CPtr9 pb, float2* __restrict__ out, int nc,
                            double boxsize, SplineDev ps) {
  const int nckz = nc/2 + 1;
  const size_t mo = blockIdx.y*((size_t) nc*nc*nckz);   // member
  for(int i = 0; i < 9; i++) pb.p[i] += mo;
  out += mo;
  const size_t row = blockIdx.x;
  const int ix = (int)(row / nc), iy = (int)(row % nc);
  for(int iz = threadIdx.x; iz < nckz; iz += blockDim.x) {
    float2 v = wbar_value(pb.p, ix, iy, iz, nc, boxsize, ps);
    if(iz == 0 || iz == nc/2) {
      const float2 m = wbar_value(pb.p, ix == 0 ? 0 : nc - ix,
                                  iy == 0 ? 0 : nc - iy, iz, nc, boxsize, ps);
      v = make_float2(0.5f*(v.x + m.x), 0.5f*(v.y - m.y));
    }
    out[row*nckz + iz] = v;
  }
}

// dense [n][n][n] <-> padded [n][n][2(n/2+1)]
__global__ void k_pad(const float* __restrict__ dense, float* __restrict__ padded,
                      int n, float scale) {
  const int ncz = 2*(n/2 + 1);
  const size_t row = blockIdx.x;
  for(int iz = threadIdx.x; iz < ncz; iz += blockDim.x)
    padded[row*ncz + iz] = iz < n ? scale*dense[row*n + iz] : 0.f;
}

__global__ void k_unpad(const float* __restrict__ padded, float* __restrict__ dense,
                        int n) {
  const int ncz = 2*(n/2 + 1);
  const size_t row = blockIdx.x;
  for(int iz = threadIdx.x; iz < n; iz += blockDim.x)
    dense[row*n + iz] = padded[row*ncz + iz];
}

int tpb_for(int m) { return m >= 256 ? 256 : (m >= 128 ? 128 : 64); }

}  // namespace

void launch_scatter3(fs2g_ctx* ctx, fs2g_particles* p, const float* fb,
                     size_t fstride, int n, float boxsize, float* g0,
                     float* g1, float* g2) {
  if(p->np_local == 0) return;
  const float dx_inv = (float) n / boxsize;
  const size_t npm = member_np(ctx, p);
  k_scatter3<<<dim3(grid_for(npm), ctx->batch), TPB, 0, ctx->stream>>>(
      p->plane(FS2G_FIELD_X, 0), p->plane(FS2G_FIELD_X, 1),
      p->plane(FS2G_FIELD_X, 2), fb, fb + fstride, fb + 2*fstride,
      npm, n, dx_inv, g0, g1, g2);
  FS2G_LAUNCHED(ctx);
}

void launch_deriv_gather(fs2g_ctx* ctx, fs2g_particles* p, const float* fb,
                         size_t fstride, const float* g0, const float* g1,
                         const float* g2, const float4* g4, const float* dbar,
                         float dfac, int n, float boxsize, float* xb,
                         size_t xstride) {
  if(p->np_local == 0) return;
  const float dx_inv = (float) n / boxsize;
  const size_t npm = member_np(ctx, p);
  k_deriv_gather<<<dim3(grid_for(npm), ctx->batch), TPB, 0, ctx->stream>>>(
      p->plane(FS2G_FIELD_X, 0), p->plane(FS2G_FIELD_X, 1),
      p->plane(FS2G_FIELD_X, 2), fb, fb ? fb + fstride : nullptr,
      fb ? fb + 2*fstride : nullptr, g0, g1, g2, g4, dbar, dfac, npm, n,
      dx_inv, xb, xb + xstride, xb + 2*xstride);
  FS2G_LAUNCHED(ctx);
}

void launch_poisson_adj_k(fs2g_ctx* ctx, const float2* G0, const float2* G1,
                          const float2* G2, float2* out, int n, float f1) {
  const size_t total = (size_t) n*n*(n/2 + 1);
  const unsigned blocks = (unsigned) std::min<size_t>((total + TPB - 1)/TPB,
                                                      (size_t) ctx->sm_count*16);
  k_poisson_adj_k<<<dim3(blocks, ctx->batch), TPB, 0, ctx->stream>>>(
      G0, G1, G2, out, n, f1);
  FS2G_LAUNCHED(ctx);
}

void launch_cola_adj(fs2g_ctx* ctx, float* xb, float* vb, float* d1b,
                     float* d2b, float* fb, size_t stride, size_t np, float K,
                     float q1, float q2, float dt, float da1, float da2) {
  if(np == 0) return;
  for(int c = 0; c < 3; c++) {
    k_cola_adj<<<grid_for(np), TPB, 0, ctx->stream>>>(
        xb + c*stride, vb + c*stride, d1b + c*stride, d2b + c*stride,
        fb + c*stride, np, K, q1, q2, dt, da1, da2);
    FS2G_LAUNCHED(ctx);
  }
}

void launch_white_to_delta(fs2g_ctx* ctx, float2* X, int nc, double boxsize,
                           SplineDev ps) {
  k_white_to_delta<<<dim3((unsigned)((size_t) nc*nc), ctx->batch),
                     tpb_for(nc/2 + 1), 0, ctx->stream>>>(X, nc, boxsize, ps);
  FS2G_LAUNCHED(ctx);
}

void launch_lpt_adj_to_mesh(fs2g_ctx* ctx, const float* xb, const float* d1b,
                            const float* d2b, size_t stride, int nc, float D1,
                            float D2, float* const p[3], float* const q[3]) {
  const size_t np = (size_t) nc*nc*nc;
  const float inv3 = (float)(1.0/((double) nc*nc*nc));
  k_lpt_adj_to_mesh<<<dim3(grid_for(np), ctx->batch), TPB, 0, ctx->stream>>>(
      xb, d1b, d2b, stride, nc, D1, D2, inv3, p[0], p[1], p[2], q[0], q[1], q[2]);
  FS2G_LAUNCHED(ctx);
}

void launch_lpt_adj_s(fs2g_ctx* ctx, float2* const pb[3], float2* out, int nc,
                      double boxsize) {
  CPtr3 a;
  for(int i = 0; i < 3; i++) a.p[i] = pb[i];
  k_lpt_adj_s<<<dim3((unsigned)((size_t) nc*nc), ctx->batch), tpb_for(nc/2 + 1),
                0, ctx->stream>>>(
      a, out, nc, boxsize);
  FS2G_LAUNCHED(ctx);
}

void launch_lpt_adj_source(fs2g_ctx* ctx, int nc, float* const ij[6],
                           const float* sbar) {
  // rows of every member (the stacked meshes are contiguous)
  k_lpt_adj_source<<<(unsigned)((size_t) nc*nc*ctx->batch), tpb_for(nc), 0,
                     ctx->stream>>>(
      nc, ij[0], ij[1], ij[2], ij[3], ij[4], ij[5], sbar);
  FS2G_LAUNCHED(ctx);
}

void launch_lpt_adj_w(fs2g_ctx* ctx, float2* const pb[9], float2* out, int nc,
                      double boxsize, SplineDev ps) {
  CPtr9 a;
  for(int i = 0; i < 9; i++) a.p[i] = pb[i];
  k_lpt_adj_w<<<dim3((unsigned)((size_t) nc*nc), ctx->batch), tpb_for(nc/2 + 1),
                0, ctx->stream>>>(
      a, out, nc, boxsize, ps);
  FS2G_LAUNCHED(ctx);
}

void launch_pad(fs2g_ctx* ctx, const float* dense, float* padded, int n,
                float scale) {
  // rows of every member: dense [batch][n][n][n] -> padded [batch][n][n][ncz]
  k_pad<<<(unsigned)((size_t) n*n*ctx->batch), tpb_for(n), 0, ctx->stream>>>(
      dense, padded, n, scale);
  FS2G_LAUNCHED(ctx);
}

void launch_unpad(fs2g_ctx* ctx, const float* padded, float* dense, int n) {
  k_unpad<<<(unsigned)((size_t) n*n*ctx->batch), tpb_for(n), 0, ctx->stream>>>(
      padded, dense, n);
  FS2G_LAUNCHED(ctx);
}

}  // namespace fs2g
