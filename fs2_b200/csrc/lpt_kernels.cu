// lpt_kernels.cu -- 2LPT initial-condition kernels for sm_100a.
//
// Restates py/lpt.cpp: the Zel'dovich displacement psi(k) from a Gaussian
// field (lpt_generate_psi_k, :276-436), its derivatives psi_ij(k)
// (lpt_compute_psi2_k, :465-505), the second-order source in real space
// (:522-535), psi2(k) (:546-586) and the particle grid (:137-211).  Mode
// values are computed in double and stored as float, as the reference does;
// the k-space kernels write each element from one thread, so the Hermitian
// pairing of the kz = 0 plane (:379-426) becomes "each element knows its
// owner column" instead of an owner writing two elements.
#include "internal.h"

namespace fs2g {

// ---------------------------------------------------------------------
// Uniform draws.  The reference draws (phase, amplitude) pairs from GSL's
// ranlxd1, reseeded per (ix, iy) column from an N-GenIC seed table.  Here
// each column has its own SplitMix64 stream (Steele, Lea & Flood 2014),
// seeded from (seed, signed kx, signed ky); draw j of the column is the j-th
// output, phase = draw 2 iz, amplitude = draw 2 iz + 1.  Keying on the
// signed wavenumber keeps a mode's draws the same at any nc that holds it.
// u = (h >> 11 + 0.5) 2^-53 lies in (0, 1), so the amplitude is never 0.
// ---------------------------------------------------------------------
__host__ __device__ __forceinline__ uint64_t sm64_mix(uint64_t z) {
  z = (z ^ (z >> 30))*0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27))*0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
constexpr uint64_t SM64_GAMMA = 0x9E3779B97F4A7C15ull;

__host__ __device__ __forceinline__ uint64_t lpt_column_state(
    uint64_t seed, int kx, int ky) {
  const uint64_t s = sm64_mix(seed + SM64_GAMMA);
  const uint64_t c = ((uint64_t)(uint32_t) kx << 32) | (uint32_t) ky;
  return sm64_mix(s ^ sm64_mix(c + 0x632BE59BD9B4E019ull));
}

__host__ __device__ __forceinline__ double u01(uint64_t h) {
  return ((double)(h >> 11) + 0.5)*(1.0/9007199254740992.0);
}

__host__ __device__ __forceinline__ void lpt_draw_pair(uint64_t col, int iz,
                                                       double* uphase,
                                                       double* uampl) {
  const uint64_t j = 2*(uint64_t) iz;
  *uphase = u01(sm64_mix(col + (j + 1)*SM64_GAMMA));
  *uampl = u01(sm64_mix(col + (j + 2)*SM64_GAMMA));
}

__host__ __device__ __forceinline__ int signed_k(int i, int nc) {
  return i < nc/2 ? i : i - nc;
}

namespace {

constexpr int TPB = 256;

__device__ __forceinline__ double lpt_kv(int i, int nc, double dk) {
  // py/lpt.cpp:333-346 and :469-482: i < nc/2 ? dk i : -dk (nc - i)
  return i < nc/2 ? dk*i : -dk*(nc - i);
}

__device__ double spline_logP(const SplineDev& s, double lk) {
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
  const double a = s.coef[lo], b = s.coef[m + lo], c = s.coef[2*m + lo],
               d = s.coef[3*m + lo];
  return a + t*(b + t*(c + t*d));
}

// psi_i(k) of one element, py/lpt.cpp:321-426.  The element is either
// written from its own column's draws or, on the kz = 0 plane, is the
// conjugate partner of an owner column.
__global__ void k_lpt_psi_k(int nc, double boxsize, uint64_t seed,
                            const double* __restrict__ u_phase,
                            const double* __restrict__ u_ampl, SplineDev ps,
                            float2* __restrict__ p0, float2* __restrict__ p1,
                            float2* __restrict__ p2) {
  const int nckz = nc/2 + 1;
  const size_t row = blockIdx.x;
  const int ix = (int)(row / nc), iy = (int)(row % nc);
  const double dk = 2.0*M_PI/boxsize;
  const double knq = nc*M_PI/boxsize;
  const double fac = pow(2*M_PI/boxsize, 1.5);
  const double fac_2pi3 = 1.0/(8.0*M_PI*M_PI*M_PI);
  for(int iz = threadIdx.x; iz < nckz; iz += blockDim.x) {
    const size_t index = row*nckz + iz;
    float2 out[3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f),
                     make_float2(0.f, 0.f)};
    bool write = true;
    int ox = ix, oy = iy;
    bool conj = false;
    if(iz == nc/2 || ix == nc/2 || iy == nc/2) write = false;       // :328
    else if(iz == 0) {
      if(ix == 0 && iy == 0) write = false;                         // :330
      else if(ix == 0) {                                             // :380-396
        if(iy >= nc/2) { oy = nc - iy; conj = true; }
      }
      else if(ix >= nc/2) {                                          // :398-423
        ox = nc - ix; oy = iy == 0 ? 0 : nc - iy; conj = true;
      }
    }
    if(write) {
      double phase, ampl;
      if(u_phase) {
        const size_t d = ((size_t) ox*nc + oy)*(nc/2) + iz;
        phase = u_phase[d]; ampl = u_ampl[d];
      }
      else {
        const uint64_t col = lpt_column_state(seed, signed_k(ox, nc),
                                              signed_k(oy, nc));
        lpt_draw_pair(col, iz, &phase, &ampl);
      }
      phase = phase*2*M_PI;                                          // :322
      double kvec[3] = {lpt_kv(ox, nc, dk), lpt_kv(oy, nc, dk),
                        lpt_kv(iz, nc, dk)};
      const double kmag2 = kvec[0]*kvec[0] + kvec[1]*kvec[1] + kvec[2]*kvec[2];
      const double kmag = sqrt(kmag2);
      if(fabs(kvec[0]) <= knq && fabs(kvec[1]) <= knq && fabs(kvec[2]) <= knq) {
        const double delta2 = -log(ampl)*fac_2pi3*exp(spline_logP(ps, log(kmag)));
        const double dkm = fac*sqrt(delta2);                          // :366
        const double sn = sin(phase), cs = cos(phase);
        for(int i = 0; i < 3; i++) {
          const double re = -kvec[i]/kmag2*dkm*sn;
          const double im = kvec[i]/kmag2*dkm*cs;
          out[i] = make_float2(__double2float_rn(re),
                               __double2float_rn(conj ? -im : im));
        }
      }
    }
    p0[index] = out[0]; p1[index] = out[1]; p2[index] = out[2];
  }
}

// psi_i(k) = i k_i/k^2 delta(k) for a given delta(k), LPT wavenumbers,
// zero on the Nyquist planes and at k = 0; Hermitian part taken on kz = 0.
__device__ __forceinline__ void psi_from_delta_one(const float2* dk_in, int ix,
                                                   int iy, int iz, int nc,
                                                   double dk, double out[6]) {
  for(int i = 0; i < 6; i++) out[i] = 0.0;
  if(ix == nc/2 || iy == nc/2 || iz == nc/2) return;
  if(ix == 0 && iy == 0 && iz == 0) return;
  const double kvec[3] = {lpt_kv(ix, nc, dk), lpt_kv(iy, nc, dk),
                          lpt_kv(iz, nc, dk)};
  const double k2 = kvec[0]*kvec[0] + kvec[1]*kvec[1] + kvec[2]*kvec[2];
  const float2 d = dk_in[((size_t) ix*nc + iy)*(nc/2 + 1) + iz];
  for(int i = 0; i < 3; i++) {
    out[2*i] = -kvec[i]/k2*(double) d.y;
    out[2*i + 1] = kvec[i]/k2*(double) d.x;
  }
}

__global__ void k_lpt_psi_from_delta(int nc, double boxsize,
                                     const float2* __restrict__ dkin,
                                     float2* __restrict__ p0,
                                     float2* __restrict__ p1,
                                     float2* __restrict__ p2) {
  const int nckz = nc/2 + 1;
  const size_t mo = blockIdx.y*((size_t) nc*nc*nckz);   // member
  dkin += mo; p0 += mo; p1 += mo; p2 += mo;
  const size_t row = blockIdx.x;
  const int ix = (int)(row / nc), iy = (int)(row % nc);
  const double dk = 2.0*M_PI/boxsize;
  for(int iz = threadIdx.x; iz < nckz; iz += blockDim.x) {
    double v[6];
    psi_from_delta_one(dkin, ix, iy, iz, nc, dk, v);
    if(iz == 0) {
      double m[6];
      psi_from_delta_one(dkin, ix == 0 ? 0 : nc - ix, iy == 0 ? 0 : nc - iy,
                         0, nc, dk, m);
      for(int i = 0; i < 3; i++) {
        v[2*i] = 0.5*(v[2*i] + m[2*i]);
        v[2*i + 1] = 0.5*(v[2*i + 1] - m[2*i + 1]);
      }
    }
    const size_t index = row*nckz + iz;
    p0[index] = make_float2(__double2float_rn(v[0]), __double2float_rn(v[1]));
    p1[index] = make_float2(__double2float_rn(v[2]), __double2float_rn(v[3]));
    p2[index] = make_float2(__double2float_rn(v[4]), __double2float_rn(v[5]));
  }
}

struct Ptr3 { float2* p[3]; };
struct Ptr6 { float2* p[6]; };
struct RPtr6 { float* p[6]; };
struct RPtr3 { float* p[3]; };

// psi_ij(k) = i k_j psi_i(k): (-Im psi_i k_j, Re psi_i k_j), py/lpt.cpp:486-502
__global__ void k_lpt_psi_ij(int nc, double boxsize, Ptr3 psi, Ptr6 out) {
  const int nckz = nc/2 + 1;
  const size_t mo = blockIdx.y*((size_t) nc*nc*nckz);   // member
  for(int i = 0; i < 3; i++) psi.p[i] += mo;
  for(int i = 0; i < 6; i++) out.p[i] += mo;
  const size_t row = blockIdx.x;
  const int ix = (int)(row / nc), iy = (int)(row % nc);
  const double dk = 2.0*M_PI/boxsize;
  const int ci[6] = {0, 0, 0, 1, 1, 2};
  const int cj[6] = {0, 1, 2, 1, 2, 2};
  for(int iz = threadIdx.x; iz < nckz; iz += blockDim.x) {
    const size_t index = row*nckz + iz;
    const double kvec[3] = {lpt_kv(ix, nc, dk), lpt_kv(iy, nc, dk),
                            lpt_kv(iz, nc, dk)};
    const float2 s[3] = {psi.p[0][index], psi.p[1][index], psi.p[2][index]};
#pragma unroll
    for(int m = 0; m < 6; m++) {
      const float2 q = s[ci[m]];
      out.p[m][index] = make_float2(
          __double2float_rn(__dmul_rn((double)(-q.y), kvec[cj[m]])),
          __double2float_rn(__dmul_rn((double) q.x, kvec[cj[m]])));
    }
  }
}

// 2LPT source, py/lpt.cpp:527-532, float in the reference's order:
// ((((p11 (p22 + p33)) + p22 p33) - p12^2) - p13^2) - p23^2
__global__ void k_lpt_source(int nc, RPtr6 ij, float* __restrict__ div) {
  const int nczr = 2*(nc/2 + 1);
  const size_t row = blockIdx.x;
  for(int iz = threadIdx.x; iz < nc; iz += blockDim.x) {
    const size_t index = row*nczr + iz;
    const float a = ij.p[0][index], b = ij.p[1][index], c = ij.p[2][index];
    const float d = ij.p[3][index], e = ij.p[4][index], f = ij.p[5][index];
    float s = __fmul_rn(a, __fadd_rn(d, f));
    s = __fadd_rn(s, __fmul_rn(d, f));
    s = __fsub_rn(s, __fmul_rn(b, b));
    s = __fsub_rn(s, __fmul_rn(c, c));
    s = __fsub_rn(s, __fmul_rn(e, e));
    div[index] = s;
  }
}

// psi2_i(k) = (S_im k_i/k^2, -S_re k_i/k^2), py/lpt.cpp:546-586.  The LPT
// wavenumber convention maps index nc/2 to -nc/2, so the result is not
// Hermitian on the kz = 0 and kz = nc/2 planes; as for the PM force, the
// Hermitian part is stored there (what an x,y-first C2R computes).
__device__ __forceinline__ void psi2_one(const float2* __restrict__ dv, int ix,
                                         int iy, int iz, int nc, double dk,
                                         double o[6]) {
  if(ix == 0 && iy == 0 && iz == 0) {
    for(int i = 0; i < 6; i++) o[i] = 0.0;
    return;
  }
  const double kvec[3] = {lpt_kv(ix, nc, dk), lpt_kv(iy, nc, dk),
                          lpt_kv(iz, nc, dk)};
  const double kmag2 = kvec[0]*kvec[0] + kvec[1]*kvec[1] + kvec[2]*kvec[2];
  const float2 s = dv[((size_t) ix*nc + iy)*(nc/2 + 1) + iz];
  for(int i = 0; i < 3; i++) {
    o[2*i] = __ddiv_rn(__dmul_rn((double) s.y, kvec[i]), kmag2);
    o[2*i + 1] = __ddiv_rn(__dmul_rn((double)(-s.x), kvec[i]), kmag2);
  }
}

__global__ void k_lpt_psi2_k(int nc, double boxsize,
                             const float2* __restrict__ div_k, Ptr3 out) {
  const int nckz = nc/2 + 1;
  const size_t mo = blockIdx.y*((size_t) nc*nc*nckz);   // member
  div_k += mo;
  for(int i = 0; i < 3; i++) out.p[i] += mo;
  const size_t row = blockIdx.x;
  const int ix = (int)(row / nc), iy = (int)(row % nc);
  const double dk = 2.0*M_PI/boxsize;
  for(int iz = threadIdx.x; iz < nckz; iz += blockDim.x) {
    double o[6];
    psi2_one(div_k, ix, iy, iz, nc, dk, o);
    float2 r[3];
    for(int i = 0; i < 3; i++)
      r[i] = make_float2(__double2float_rn(o[2*i]),
                         __double2float_rn(o[2*i + 1]));
    if(iz == 0 || iz == nc/2) {
      double m[6];
      psi2_one(div_k, ix == 0 ? 0 : nc - ix, iy == 0 ? 0 : nc - iy, iz, nc,
               dk, m);
      for(int i = 0; i < 3; i++) {
        const float mre = __double2float_rn(m[2*i]);
        const float mim = __double2float_rn(m[2*i + 1]);
        r[i] = make_float2(__fmul_rn(0.5f, __fadd_rn(r[i].x, mre)),
                           __fmul_rn(0.5f, __fsub_rn(r[i].y, mim)));
      }
    }
    const size_t index = row*nckz + iz;
    for(int i = 0; i < 3; i++) out.p[i][index] = r[i];
  }
}

// the particle grid, py/lpt.cpp:182-211, one thread per particle
__global__ void __launch_bounds__(TPB)
k_lpt_particles(int nc, float dx, float offset, double nmesh3_inv, RPtr3 psi,
                RPtr3 psi2, float D1, float D2, float Dv, float D2v,
                size_t stride, float* __restrict__ planes,
                uint64_t* __restrict__ id) {
  // member blockIdx.y: its particles start at blockIdx.y np, its meshes
  // blockIdx.y nc^2 nczr floats in; ids count from 1 in every member
  const size_t np = (size_t) nc*nc*nc;
  const size_t il = blockIdx.x*(size_t)blockDim.x + threadIdx.x;
  if(il >= np) return;
  const int nczr = 2*(nc/2 + 1);
  const size_t mo = blockIdx.y*((size_t) nc*nc*nczr);
  for(int k = 0; k < 3; k++) { psi.p[k] += mo; psi2.p[k] += mo; }
  planes += blockIdx.y*np;
  id += blockIdx.y*np;
  const size_t ip = il;
  const size_t iz = ip % nc, t = ip / nc;
  const size_t iy = t % nc, ix = t / nc;
  const size_t index = (ix*nc + iy)*nczr + iz;
  const size_t q[3] = {ix, iy, iz};
#pragma unroll
  for(int k = 0; k < 3; k++) {
    const float xq = __fmul_rn(__fadd_rn((float) q[k], offset), dx);
    const float dis = psi.p[k][index];
    const float dis2 = __double2float_rn(__dmul_rn(nmesh3_inv,
                                                   (double) psi2.p[k][index]));
    const float x = __fadd_rn(__fadd_rn(xq, __fmul_rn(D1, dis)),
                              __fmul_rn(D2, dis2));
    const float v = __fadd_rn(__fmul_rn(Dv, dis), __fmul_rn(D2v, dis2));
    planes[(size_t)(0 + k)*stride + ip] = x;
    planes[(size_t)(3 + k)*stride + ip] = v;
    planes[(size_t)(6 + k)*stride + ip] = dis;
    planes[(size_t)(9 + k)*stride + ip] = dis2;
    planes[(size_t)(12 + k)*stride + ip] = 0.0f;   // force (calloc'd)
  }
  id[ip] = (uint64_t) ip + 1;
}

int lpt_tpb(int nckz) { return nckz >= 256 ? 256 : (nckz >= 128 ? 128 : 64); }

}  // namespace

// ---------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------
void launch_lpt_psi_k(fs2g_ctx* ctx, int nc, double boxsize,
                      unsigned long long seed, const double* u_phase,
                      const double* u_ampl, SplineDev ps, float2* psi0,
                      float2* psi1, float2* psi2) {
  k_lpt_psi_k<<<(unsigned)((size_t) nc*nc), lpt_tpb(nc/2 + 1), 0, ctx->stream>>>(
      nc, boxsize, (uint64_t) seed, u_phase, u_ampl, ps, psi0, psi1, psi2);
  FS2G_LAUNCHED(ctx);
}

void launch_lpt_psi_from_delta(fs2g_ctx* ctx, int nc, double boxsize,
                               const float2* delta_k, float2* psi0,
                               float2* psi1, float2* psi2) {
  k_lpt_psi_from_delta<<<dim3((unsigned)((size_t) nc*nc), ctx->batch),
                         lpt_tpb(nc/2 + 1), 0, ctx->stream>>>(
      nc, boxsize, delta_k, psi0, psi1, psi2);
  FS2G_LAUNCHED(ctx);
}

void launch_lpt_psi_ij(fs2g_ctx* ctx, int nc, double boxsize,
                       float2* const psi[3], float2* const out[6]) {
  Ptr3 a; Ptr6 b;
  for(int i = 0; i < 3; i++) a.p[i] = psi[i];
  for(int i = 0; i < 6; i++) b.p[i] = out[i];
  k_lpt_psi_ij<<<dim3((unsigned)((size_t) nc*nc), ctx->batch),
                 lpt_tpb(nc/2 + 1), 0, ctx->stream>>>(nc, boxsize, a, b);
  FS2G_LAUNCHED(ctx);
}

void launch_lpt_source(fs2g_ctx* ctx, int nc, float* const ij[6], float* div) {
  RPtr6 a;
  for(int i = 0; i < 6; i++) a.p[i] = ij[i];
  // rows of every member (the stacked meshes are contiguous)
  k_lpt_source<<<(unsigned)((size_t) nc*nc*ctx->batch), lpt_tpb(nc), 0,
                 ctx->stream>>>(nc, a, div);
  FS2G_LAUNCHED(ctx);
}

void launch_lpt_psi2_k(fs2g_ctx* ctx, int nc, double boxsize,
                       const float2* div_k, float2* const out[3]) {
  Ptr3 a;
  for(int i = 0; i < 3; i++) a.p[i] = out[i];
  k_lpt_psi2_k<<<dim3((unsigned)((size_t) nc*nc), ctx->batch),
                 lpt_tpb(nc/2 + 1), 0, ctx->stream>>>(nc, boxsize, div_k, a);
  FS2G_LAUNCHED(ctx);
}

void launch_lpt_particles(fs2g_ctx* ctx, fs2g_particles* p, int nc,
                          double boxsize, float offset,
                          float* const psi[3], float* const psi2[3],
                          float D1, float D2, float Dv, float D2v) {
  RPtr3 a, b;
  for(int i = 0; i < 3; i++) { a.p[i] = psi[i]; b.p[i] = psi2[i]; }
  const size_t np = (size_t) nc*nc*nc;
  const float dx = (float)(boxsize/nc);                  // py/lpt.cpp:144
  const double nmesh3_inv = 1.0/pow((double) nc, 3.0);   // py/lpt.cpp:147
  k_lpt_particles<<<dim3((unsigned)((np + TPB - 1)/TPB), ctx->batch), TPB, 0,
                    ctx->stream>>>(
      nc, dx, offset, nmesh3_inv, a, b, D1, D2, Dv, D2v, p->stride,
      p->d_planes, p->d_id);
  FS2G_LAUNCHED(ctx);
}

// host generation of the draws (same integer arithmetic as the kernel)
void lpt_draws_host(int nc, unsigned long long seed, double* u_phase,
                    double* u_ampl) {
  const int nzd = nc/2;
  for(int ix = 0; ix < nc; ix++)
    for(int iy = 0; iy < nc; iy++) {
      const uint64_t col = lpt_column_state((uint64_t) seed, signed_k(ix, nc),
                                            signed_k(iy, nc));
      for(int iz = 0; iz < nzd; iz++) {
        const size_t d = ((size_t) ix*nc + iy)*nzd + iz;
        lpt_draw_pair(col, iz, u_phase + d, u_ampl + d);
      }
    }
}

}  // namespace fs2g
