// fft_pipeline.cu -- the PM Poisson solve as five fused FFT passes (sm_100a).
//
// Replaces R2C + 3 x (k-space force + C2R) of py/pm.cpp:431-508 for meshes
// with n a power of two, 64 <= n <= 1024.  The reference (and a library FFT)
// moves the mesh through HBM four times per transform plus once per k-space
// pass; here the transforms are split by axis and fused across the
// boundaries between them:
//
//   FZ  R2C along z               real delta(x,y,z) -> A(x,y,kz)
//   FY  forward along y           A -> A(x,ky,kz)                 (in place)
//   XX  forward along x, Green's function, inverse along x:
//         G = i f1/k^2 delta(k),  H = k_x G   ->  C = IFx[G], B = IFx[H]
//   IY  inverse along y:  A = IFy[C], D = IFy[k_y C] (f_y), B = IFy[B] (f_x)
//   IZ  C2R along z:  f_x <- B,  f_y <- D,  f_z <- k_z A, written
//       interleaved as (f_x, f_y, f_z, 0) per cell, the layout the gather
//       reads with one 16-byte load per CIC corner
//
// delta(k) is never written to HBM (unless asked for), and the k-space
// multiply costs no pass of its own.  The C2R along z ignores the imaginary
// parts of the kz = 0 and kz = n/2 bins, which is what FFTW's and
// pocketfft's multi-dimensional C2R do; on the reference's spectrum (not
// Hermitian on those planes, +n/2 Nyquist convention) that is the Hermitian
// projection the cuFFT path applies explicitly.
//
// FFT core: a warp transforms one length-L = 32 R sequence held in shared
// memory with one pad slot per 32 elements: an R-point DFT per lane over
// elements l + 32 m, a twiddle, then 32-point DFTs over the lanes (Cooley-
// Tukey L = R x 32), all radix-2 in registers.  Tile passes (FY, XX, IY) keep
// 8 columns of 8 consecutive kz, one warp per column, column-major in shared
// memory.  Complex intermediates use a row pitch PC = n/2+1 rounded up to 8,
// so that every row starts 64-byte aligned.
#include "internal.h"

namespace fs2g {
namespace {

constexpr int TILE_W = 8;        // kz columns per tile: pitch granularity

// exp(-2 pi i t / 32), t = 0..31, as literals so that the unrolled
// butterflies multiply by immediates (t = 0 and t = 8 are special-cased)
__device__ static const float kW32re[32] = {
  1.0f, 9.807852804e-01f, 9.238795325e-01f, 8.314696123e-01f,
  7.071067812e-01f, 5.555702330e-01f, 3.826834324e-01f, 1.950903220e-01f,
  0.0f, -1.950903220e-01f, -3.826834324e-01f, -5.555702330e-01f,
  -7.071067812e-01f, -8.314696123e-01f, -9.238795325e-01f, -9.807852804e-01f,
  -1.0f, -9.807852804e-01f, -9.238795325e-01f, -8.314696123e-01f,
  -7.071067812e-01f, -5.555702330e-01f, -3.826834324e-01f, -1.950903220e-01f,
  0.0f, 1.950903220e-01f, 3.826834324e-01f, 5.555702330e-01f,
  7.071067812e-01f, 8.314696123e-01f, 9.238795325e-01f, 9.807852804e-01f};
__device__ static const float kW32im[32] = {
  0.0f, -1.950903220e-01f, -3.826834324e-01f, -5.555702330e-01f,
  -7.071067812e-01f, -8.314696123e-01f, -9.238795325e-01f, -9.807852804e-01f,
  -1.0f, -9.807852804e-01f, -9.238795325e-01f, -8.314696123e-01f,
  -7.071067812e-01f, -5.555702330e-01f, -3.826834324e-01f, -1.950903220e-01f,
  0.0f, 1.950903220e-01f, 3.826834324e-01f, 5.555702330e-01f,
  7.071067812e-01f, 8.314696123e-01f, 9.238795325e-01f, 9.807852804e-01f,
  1.0f, 9.807852804e-01f, 9.238795325e-01f, 8.314696123e-01f,
  7.071067812e-01f, 5.555702330e-01f, 3.826834324e-01f, 1.950903220e-01f};

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y*b.y), fmaf(a.x, b.y, a.y*b.x));
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
// complex add / subtract as one packed sm_100 instruction (add.rn.f32x2,
// sub.rn.f32x2): each lane is rounded to nearest as the scalar add is, in
// half the issue slots.  Used by the XX pass only: packing every pass's
// butterflies made XX 7% faster but FZ 15% and IY 10% slower.
__device__ __forceinline__ float2 padd(float2 a, float2 b) {
  float2 r;
  asm("{\n\t.reg .b64 pa, pb, pd;\n\t"
      "mov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t"
      "add.rn.f32x2 pd, pa, pb;\n\tmov.b64 {%0, %1}, pd;\n\t}"
      : "=f"(r.x), "=f"(r.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
__device__ __forceinline__ float2 psub(float2 a, float2 b) {
  float2 r;
  asm("{\n\t.reg .b64 pa, pb, pd;\n\t"
      "mov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t"
      "sub.rn.f32x2 pd, pa, pb;\n\tmov.b64 {%0, %1}, pd;\n\t}"
      : "=f"(r.x), "=f"(r.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
template<bool INV> __device__ __forceinline__ float2 tw_dir(float2 w) {
  return INV ? cconj(w) : w;
}

__host__ __device__ constexpr int ilog2(int x) { return x <= 1 ? 0 : 1 + ilog2(x >> 1); }
__host__ __device__ constexpr int bitrev(int x, int bits) {
  int r = 0;
  for(int i = 0; i < bits; i++) { r = (r << 1) | ((x >> i) & 1); }
  return r;
}

// In-register radix-2 decimation-in-frequency DFT of R points (natural order
// in, bit-reversed order out): afterwards X[k] = v[bitrev(k)].  PK: the
// butterflies' adds packed (padd / psub), same results.
template<int R, bool INV, bool PK = false>
__device__ __forceinline__ void dif(float2* v) {
#pragma unroll
  for(int s = R/2; s >= 1; s >>= 1) {
#pragma unroll
    for(int i = 0; i < R; i += 2*s) {
#pragma unroll
      for(int j = 0; j < s; j++) {
        const float2 a = v[i + j], b = v[i + j + s];
        v[i + j] = PK ? padd(a, b) : cadd(a, b);
        const float2 d = PK ? psub(a, b) : csub(a, b);
        const int t = j*(32/(2*s));                 // omega_32^t
        if(t == 0) v[i + j + s] = d;
        else if(t == 8)                             // -i (forward), +i (inverse)
          v[i + j + s] = INV ? make_float2(-d.y, d.x) : make_float2(d.y, -d.x);
        else
          v[i + j + s] = cmul(d, tw_dir<INV>(make_float2(kW32re[t], kW32im[t])));
      }
    }
  }
}

__device__ __forceinline__ int pidx(int e) { return e + (e >> 5); }

// Warp FFT of length L = 32 R in place on a padded shared-memory column
// (element e at col[pidx(e)]), natural order in and out.  twL(j) must return
// exp(-2 pi i j / L).  Unnormalised; INV uses exp(+...).
template<int R, bool INV, bool PK = false, class TW>
__device__ __forceinline__ void warp_fft(float2* col, TW twL) {
  const int l = threadIdx.x & 31;
  constexpr int RB = ilog2(R);
  {
    float2 v[R];
#pragma unroll
    for(int m = 0; m < R; m++) v[m] = col[pidx(l + 32*m)];
    if(R > 1) dif<R, INV, PK>(v);
#pragma unroll
    for(int k1 = 0; k1 < R; k1++) {
      float2 y = v[bitrev(k1, RB)];
      if(k1 > 0 && l > 0) y = cmul(y, tw_dir<INV>(twL(l*k1)));
      col[pidx(l + 32*k1)] = y;
    }
  }
  __syncwarp();
  float2 w[32];
  if(l < R) {
#pragma unroll
    for(int j = 0; j < 32; j++) w[j] = col[pidx(32*l + j)];
  }
  __syncwarp();
  if(l < R) {
    dif<32, INV, PK>(w);
#pragma unroll
    for(int k2 = 0; k2 < 32; k2++) col[pidx(l + R*k2)] = w[bitrev(k2, 5)];
  }
  __syncwarp();
}

// B = 32/R sequences of length L = 32 R per warp (R < 32), sequence s at
// base + s*seq: step 1 runs one R-point DFT per lane per sequence, step 3 one
// 32-point DFT per lane (lane l: sequence l / R, k1 = l % R), so every lane
// works in both steps.  For R = 32 this is warp_fft.
template<int R, bool INV, class TW>
__device__ __forceinline__ void warp_fft_multi(float2* base, int seq, TW twL) {
  constexpr int B = 32/R;
  constexpr int RB = ilog2(R);
  const int l = threadIdx.x & 31;
#pragma unroll 1
  for(int sq = 0; sq < B; sq++) {
    float2* col = base + sq*seq;
    float2 v[R];
#pragma unroll
    for(int m = 0; m < R; m++) v[m] = col[pidx(l + 32*m)];
    if(R > 1) dif<R, INV>(v);
#pragma unroll
    for(int k1 = 0; k1 < R; k1++) {
      float2 y = v[bitrev(k1, RB)];
      if(k1 > 0 && l > 0) y = cmul(y, tw_dir<INV>(twL(l*k1)));
      col[pidx(l + 32*k1)] = y;
    }
  }
  __syncwarp();
  const int sq = l / R, k1 = l % R;
  float2* col = base + sq*seq;
  float2 w[32];
#pragma unroll
  for(int j = 0; j < 32; j++) w[j] = col[pidx(32*k1 + j)];
  __syncwarp();
  dif<32, INV>(w);
#pragma unroll
  for(int k2 = 0; k2 < 32; k2++) col[pidx(k1 + R*k2)] = w[bitrev(k2, 5)];
  __syncwarp();
}

// table access: tw[j*stride] = exp(-2 pi i j*stride / NT)
struct Tw {
  const float2* __restrict__ t; int stride;
  __device__ __forceinline__ float2 operator()(int j) const { return __ldg(t + j*stride); }
};

// --------------------------------------------------------------------
// FZ: R2C along z.  One warp per (x, y) row; L = n/2.
// --------------------------------------------------------------------
constexpr int ROW_WARPS = 4;     // FZ / IZ: warps per block

template<int R>
__global__ void __launch_bounds__(32*ROW_WARPS)
k_fz(const float* __restrict__ in, float2* __restrict__ out, int n, int pc,
     const float2* __restrict__ tw) {
  constexpr int L = 32*R, B = 32/R, SEQ = L + L/32 + 2;
  __shared__ float2 sm[ROW_WARPS][B*SEQ];
  const int warp = threadIdx.x >> 5, l = threadIdx.x & 31;
  const size_t row0 = ((size_t) blockIdx.x*ROW_WARPS + warp)*B;   // B rows per warp
  if(row0 >= (size_t) n*n) return;
  float2* base = sm[warp];
  const int ncz = n + 2;
#pragma unroll
  for(int sq = 0; sq < B; sq++) {
    const float2* src = reinterpret_cast<const float2*>(in + (row0 + sq)*ncz);
#pragma unroll
    for(int m = 0; m < R; m++) base[sq*SEQ + pidx(l + 32*m)] = src[l + 32*m];
  }
  __syncwarp();
  warp_fft_multi<R, false>(base, SEQ, Tw{tw, 2});          // length L = n/2
  // X_k = (Z_k + conj Z_{L-k})/2 - i W^k (Z_k - conj Z_{L-k})/2, k = 0..L
#pragma unroll 1
  for(int sq = 0; sq < B; sq++) {
    const float2* col = base + sq*SEQ;
    float2* dst = out + (row0 + sq)*pc;
    for(int k = l; k <= L; k += 32) {
      const float2 zk = col[pidx(k == L ? 0 : k)];
      const float2 zc = cconj(col[pidx(k == 0 ? 0 : L - k)]);
      const float2 e = make_float2(0.5f*(zk.x + zc.x), 0.5f*(zk.y + zc.y));
      const float2 d = make_float2(0.5f*(zk.x - zc.x), 0.5f*(zk.y - zc.y));
      const float2 w = k == L ? make_float2(-1.f, 0.f) : __ldg(tw + k);   // W^k
      const float2 wd = cmul(w, d);                  // -i * w * d below
      dst[k] = make_float2(e.x + wd.y, e.y - wd.x);
    }
  }
}

// --------------------------------------------------------------------
// tile load / store: TILE_W consecutive kz of `len` rows at row stride
// `rs` (complex elements), into column-major padded shared memory
// --------------------------------------------------------------------
template<int L>
struct TileSm { static constexpr int CP = L + L/32 + 4; };

// one thread moves two consecutive kz (16 bytes); rows are 64-byte aligned
// All of a thread's 16-byte loads are issued before any shared store, so
// that each thread keeps L*TILE_W/(2 NT) loads in flight.
template<int L, int NT, int W>
__device__ __forceinline__ void tile_load(float2* sm, const float2* __restrict__ g,
                                          size_t rs) {
  constexpr int CP = TileSm<L>::CP;
  constexpr int TOTAL = L*W/2;
  constexpr int ITEMS = (TOTAL + NT - 1)/NT;
  constexpr int CH = ITEMS < 8 ? ITEMS : 8;       // loads in flight per thread
#pragma unroll 1
  for(int i0 = 0; i0 < ITEMS; i0 += CH) {
    float4 v[CH];
#pragma unroll
    for(int i = 0; i < CH; i++) {
      const int t = threadIdx.x + (i0 + i)*NT;
      const int e = t / (W/2), w = 2*(t % (W/2));
      if(TOTAL % NT == 0 || t < TOTAL)
        v[i] = __ldg(reinterpret_cast<const float4*>(g + (size_t) e*rs + w));
    }
#pragma unroll
    for(int i = 0; i < CH; i++) {
      const int t = threadIdx.x + (i0 + i)*NT;
      const int e = t / (W/2), w = 2*(t % (W/2));
      if(TOTAL % NT == 0 || t < TOTAL) {
        sm[w*CP + pidx(e)] = make_float2(v[i].x, v[i].y);
        sm[(w + 1)*CP + pidx(e)] = make_float2(v[i].z, v[i].w);
      }
    }
  }
}

template<int L, int NT, int W>
__device__ __forceinline__ void tile_store(const float2* sm, float2* __restrict__ g,
                                           size_t rs) {
  constexpr int CP = TileSm<L>::CP;
  constexpr int TOTAL = L*W/2;
  constexpr int ITEMS = (TOTAL + NT - 1)/NT;
#pragma unroll
  for(int i = 0; i < ITEMS; i++) {
    const int t = threadIdx.x + i*NT;
    const int e = t / (W/2), w = 2*(t % (W/2));
    if(!(TOTAL % NT == 0 || t < TOTAL)) continue;
    const float2 a = sm[w*CP + pidx(e)], b = sm[(w + 1)*CP + pidx(e)];
    *reinterpret_cast<float4*>(g + (size_t) e*rs + w) = make_float4(a.x, a.y, b.x, b.y);
  }
}

// --------------------------------------------------------------------
// FY: forward FFT along y, in place.  Tile (x, kz block).
// --------------------------------------------------------------------
template<int R, int W>
__global__ void __launch_bounds__(32*W)
k_fy(float2* __restrict__ a, int n, int pc, const float2* __restrict__ tw) {
  constexpr int L = 32*R, CP = TileSm<L>::CP, NT = 32*W;
  extern __shared__ float2 sm[];
  const int tiles_z = pc/W;
  const int x = blockIdx.x / tiles_z, kz0 = (blockIdx.x % tiles_z)*W;
  float2* g = a + (size_t) x*n*pc + kz0;
  tile_load<L, NT, W>(sm, g, pc);
  __syncthreads();
  warp_fft<R, false>(sm + (threadIdx.x >> 5)*CP, Tw{tw, 1});
  __syncthreads();
  tile_store<L, NT, W>(sm, g, pc);
}

// --------------------------------------------------------------------
// XX: forward along x, Green's function, inverse along x.  Tile (ky, kz
// block).  k_i = i <= n/2 ? i : i - n (x, y), k_z = kz (py/pm.cpp:483-495);
// G = i (f1/k^2) delta, H = i (f1/k^2) k_x delta, 0 at k = 0.
// --------------------------------------------------------------------
// XX and IY: two tiles of W columns, 2 W warps.  XX reads a, writes
// IFx[G] to c and IFx[H] to b.
template<int R, int W>
__global__ void __launch_bounds__(64*W)
k_xx(const float2* __restrict__ a, float2* __restrict__ b,
     float2* __restrict__ c, float2* __restrict__ dk_out, int n, int pc,
     float f1, const float2* __restrict__ tw) {
  constexpr int L = 32*R, CP = TileSm<L>::CP, NT = 64*W;
  extern __shared__ float2 sm[];     // tile 1 (columns 0..W-1): G; tile 2: H
  const int tiles_z = pc/W;
  const int ky = blockIdx.x / tiles_z, kz0 = (blockIdx.x % tiles_z)*W;
  const size_t rs = (size_t) n*pc;
  const float2* ga = a + (size_t) ky*pc + kz0;
  float2* gb = b + (size_t) ky*pc + kz0;
  float2* gc = c + (size_t) ky*pc + kz0;
  const int warp = threadIdx.x >> 5, l = threadIdx.x & 31;
  float2* col = sm + warp*CP;        // warps W..2W-1: their H column
  tile_load<L, NT, W>(sm, ga, rs);
  __syncthreads();
  if(warp < W) warp_fft<R, false, true>(col, Tw{tw, 1});
  __syncthreads();
  if(dk_out) {
    tile_store<L, NT, W>(sm, dk_out + (size_t) ky*pc + kz0, rs);
    __syncthreads();
  }
  if(warp < W) {
    // Green's function at (kx = l + 32 m, ky, kz0 + warp)
    float2* colh = sm + (W + warp)*CP;
    const int kz = kz0 + warp;
    const float fy = (float)(ky <= n/2 ? ky : ky - n);
    const float fz = (float) kz;
#pragma unroll 4
    for(int m = 0; m < R; m++) {
      const int kx = l + 32*m;
      const float fx = (float)(kx <= n/2 ? kx : kx - n);
      const float ksq = fx*fx + fy*fy + fz*fz;
      const float2 d = col[pidx(kx)];
      float2 g2 = make_float2(0.f, 0.f), h2 = make_float2(0.f, 0.f);
      if(!(ksq == 0.0f || kz > n/2)) {
        const float g = f1/ksq;
        g2 = make_float2(-g*d.y, g*d.x);
        const float f2 = g*fx;
        h2 = make_float2(-f2*d.y, f2*d.x);
      }
      col[pidx(kx)] = g2;
      colh[pidx(kx)] = h2;
    }
  }
  __syncthreads();
  warp_fft<R, true, true>(col, Tw{tw, 1});
  __syncthreads();
  tile_store<L, NT, W>(sm, gc, rs);
  tile_store<L, NT, W>(sm + W*CP, gb, rs);
}

// --------------------------------------------------------------------
// IY: inverse along y.  Tile (x, kz block).  A <- IFy[C]; D <- IFy[k_y C];
// B <- IFy[B].
// --------------------------------------------------------------------
template<int R, int W>
__global__ void __launch_bounds__(64*W)
k_iy(float2* __restrict__ a, float2* __restrict__ b,
     const float2* __restrict__ c, float2* __restrict__ d, int n, int pc,
     const float2* __restrict__ tw) {
  constexpr int L = 32*R, CP = TileSm<L>::CP, NT = 64*W;
  extern __shared__ float2 sm[];     // tile 1: A, tile 2: k_y A, then B
  const int tiles_z = pc/W;
  const int x = blockIdx.x / tiles_z, kz0 = (blockIdx.x % tiles_z)*W;
  const size_t off = (size_t) x*n*pc + kz0;
  const int warp = threadIdx.x >> 5, l = threadIdx.x & 31;
  float2* col = sm + warp*CP;
  tile_load<L, NT, W>(sm, c + off, pc);
  __syncthreads();
  if(warp < W) {
    float2* col2 = sm + (W + warp)*CP;
#pragma unroll 4
    for(int m = 0; m < R; m++) {
      const int ky = l + 32*m;
      const float fy = (float)(ky <= n/2 ? ky : ky - n);
      const float2 v = col[pidx(ky)];
      col2[pidx(ky)] = make_float2(fy*v.x, fy*v.y);
    }
  }
  __syncthreads();
  warp_fft<R, true>(col, Tw{tw, 1});
  __syncthreads();
  tile_store<L, NT, W>(sm, a + off, pc);
  tile_store<L, NT, W>(sm + W*CP, d + off, pc);
  __syncthreads();
  tile_load<L, NT, W>(sm + W*CP, b + off, pc);
  __syncthreads();
  if(warp >= W) warp_fft<R, true>(col, Tw{tw, 1});
  __syncthreads();
  tile_store<L, NT, W>(sm + W*CP, b + off, pc);
}

// --------------------------------------------------------------------
// Tensor memory helpers (sm_100a).  A block allocates TMEM columns with
// tcgen05.alloc from one warp; warp w of the block may touch only lanes
// 32 (w % 4) .. 32 (w % 4) + 31, so each warp keeps its lanes' data in its
// own quarter.  Addresses: lane << 16 | column.
// --------------------------------------------------------------------
__device__ __forceinline__ void tmem_alloc(uint32_t* smem_dst, int ncols) {
  const uint32_t dst = (uint32_t) __cvta_generic_to_shared(smem_dst);
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
               :: "r"(dst), "r"(ncols) : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, int ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
               :: "r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tmem_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tmem_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// this thread's 64 floats -> columns taddr .. taddr + 63 of its lane
__device__ __forceinline__ void tmem_st64(uint32_t taddr, const float (&v)[64]) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x64.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32, %33, %34, %35, %36, %37, %38, %39, %40, %41, %42, %43, %44, %45, %46, %47, %48, %49, %50, %51, %52, %53, %54, %55, %56, %57, %58, %59, %60, %61, %62, %63, %64};"
      :: "r"(taddr),
      "r"(__float_as_uint(v[0])),
      "r"(__float_as_uint(v[1])),
      "r"(__float_as_uint(v[2])),
      "r"(__float_as_uint(v[3])),
      "r"(__float_as_uint(v[4])),
      "r"(__float_as_uint(v[5])),
      "r"(__float_as_uint(v[6])),
      "r"(__float_as_uint(v[7])),
      "r"(__float_as_uint(v[8])),
      "r"(__float_as_uint(v[9])),
      "r"(__float_as_uint(v[10])),
      "r"(__float_as_uint(v[11])),
      "r"(__float_as_uint(v[12])),
      "r"(__float_as_uint(v[13])),
      "r"(__float_as_uint(v[14])),
      "r"(__float_as_uint(v[15])),
      "r"(__float_as_uint(v[16])),
      "r"(__float_as_uint(v[17])),
      "r"(__float_as_uint(v[18])),
      "r"(__float_as_uint(v[19])),
      "r"(__float_as_uint(v[20])),
      "r"(__float_as_uint(v[21])),
      "r"(__float_as_uint(v[22])),
      "r"(__float_as_uint(v[23])),
      "r"(__float_as_uint(v[24])),
      "r"(__float_as_uint(v[25])),
      "r"(__float_as_uint(v[26])),
      "r"(__float_as_uint(v[27])),
      "r"(__float_as_uint(v[28])),
      "r"(__float_as_uint(v[29])),
      "r"(__float_as_uint(v[30])),
      "r"(__float_as_uint(v[31])),
      "r"(__float_as_uint(v[32])),
      "r"(__float_as_uint(v[33])),
      "r"(__float_as_uint(v[34])),
      "r"(__float_as_uint(v[35])),
      "r"(__float_as_uint(v[36])),
      "r"(__float_as_uint(v[37])),
      "r"(__float_as_uint(v[38])),
      "r"(__float_as_uint(v[39])),
      "r"(__float_as_uint(v[40])),
      "r"(__float_as_uint(v[41])),
      "r"(__float_as_uint(v[42])),
      "r"(__float_as_uint(v[43])),
      "r"(__float_as_uint(v[44])),
      "r"(__float_as_uint(v[45])),
      "r"(__float_as_uint(v[46])),
      "r"(__float_as_uint(v[47])),
      "r"(__float_as_uint(v[48])),
      "r"(__float_as_uint(v[49])),
      "r"(__float_as_uint(v[50])),
      "r"(__float_as_uint(v[51])),
      "r"(__float_as_uint(v[52])),
      "r"(__float_as_uint(v[53])),
      "r"(__float_as_uint(v[54])),
      "r"(__float_as_uint(v[55])),
      "r"(__float_as_uint(v[56])),
      "r"(__float_as_uint(v[57])),
      "r"(__float_as_uint(v[58])),
      "r"(__float_as_uint(v[59])),
      "r"(__float_as_uint(v[60])),
      "r"(__float_as_uint(v[61])),
      "r"(__float_as_uint(v[62])),
      "r"(__float_as_uint(v[63]))
      : "memory");
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}
// columns taddr .. taddr + 15 of this thread's lane -> r
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr) : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// r -> columns taddr .. taddr + 15 of this thread's lane
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t (&r)[16]) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16};"
      :: "r"(taddr), "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]),
         "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
      : "memory");
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

// cells p[0] and p[1] (32 bytes, p 32-byte aligned) in one 256-bit store:
// a lane's two adjacent cells become whole 32-byte sectors (two 16-byte
// stores from lanes 32 bytes apart left every sector half written per
// instruction; IZ 6.2 -> 5.3 ms at n = 1024)
__device__ __forceinline__ void st_global_v8(float4* p, float4 a, float4 b) {
  asm volatile("st.global.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};"
               :: "l"(p), "f"(a.x), "f"(a.y), "f"(a.z), "f"(a.w),
                  "f"(b.x), "f"(b.y), "f"(b.z), "f"(b.w) : "memory");
}

// --------------------------------------------------------------------
// Register-direct tile passes for n = 1024 (L = 32 x 32), 8 columns per
// tile, 256 threads.  Thread (c, s), c = tid % 8, s = tid / 8, loads the
// 32 elements s + 32 m (m = 0..31) of column c straight from HBM: one warp
// instruction reads four 64-byte row segments.  Step A (32-point DFT over m,
// twiddle W_L^{s k1}) runs in registers, one shared-memory transposition
// Y[c][s][k1] -> thread (c, k1) follows, and step B (32-point DFT over s)
// leaves X[k1 + 32 k2] in the registers of thread (c, k1), which stores it
// straight to HBM.  Shared memory is touched once per element and
// transform (write + read), conflict-free with word strides 1058 (column)
// and 33 (row); the whole tile's loads are in flight at once and no
// registers stage them.  Same decomposition and operation order as
// warp_fft, so the results are bitwise those of the tile kernels above.
// --------------------------------------------------------------------
constexpr int RD_W = 8, RD_NT = 256, RD_SC = 1058, RD_SS = 33;
constexpr int RD_N = 1024, RD_PC = ((RD_N/2 + 1) + TILE_W - 1)/TILE_W*TILE_W;
constexpr size_t RD_SMEM = (size_t) RD_W*RD_SC*sizeof(float2);

// step A on v[m] (natural order in): DFT over m, then W_L^{s k1}; leaves
// Y[k1] in v[bitrev(k1)] and writes it to buf[c][s][k1]
template<bool INV, bool PK = false>
__device__ __forceinline__ void rd_step_a(float2 (&v)[32], int c, int s,
                                          float2* buf,
                                          const float2* __restrict__ tw) {
  dif<32, INV, PK>(v);
#pragma unroll
  for(int k1 = 0; k1 < 32; k1++) {
    float2 y = v[bitrev(k1, 5)];
    if(k1 > 0 && s > 0) y = cmul(y, tw_dir<INV>(__ldg(tw + s*k1)));
    buf[c*RD_SC + s*RD_SS + k1] = y;
  }
}

// step B: thread (c, k1 = s) reads buf[c][j][s], j = 0..31, and runs the DFT
// over j; afterwards X[s + 32 k2] = w[bitrev(k2)]
template<bool INV, bool PK = false>
__device__ __forceinline__ void rd_step_b(float2 (&w)[32], int c, int s,
                                          const float2* buf) {
#pragma unroll
  for(int j = 0; j < 32; j++) w[j] = buf[c*RD_SC + j*RD_SS + s];
  dif<32, INV, PK>(w);
}

// hint: bring the 128-byte line holding p into L2
__device__ __forceinline__ void prefetch_l2(const void* p) {
  asm volatile("prefetch.global.L2 [%0];" :: "l"(p));
}

// The tile passes below are latency-bound at two blocks per SM: each block
// loads its tile, transforms it and stores it with nothing of its own to
// overlap.  So each block first prefetches into L2 the tile of block
// blockIdx.x + la (la = one block per SM: the block that starts about half
// a wave later), whose loads then hit L2.  Measured at n = 1024: FY 1.77 ->
// 1.45 ms, IY 4.78 -> 4.09 ms; a whole wave ahead gains less, and XX (more
// arithmetic per byte) gains nothing.
// FY, n = 1024: forward along y in place.  Tile (x, kz block).
__global__ void __launch_bounds__(RD_NT, 2)
k_fy_rd(float2* __restrict__ a, const float2* __restrict__ tw, unsigned la) {
  constexpr int n = RD_N, pc = RD_PC;
  extern __shared__ float2 sm[];
  const int tiles_z = pc/RD_W;
  const int x = blockIdx.x / tiles_z, kz0 = (blockIdx.x % tiles_z)*RD_W;
  const int c = threadIdx.x & 7, s = threadIdx.x >> 3;
  float2* g = a + (size_t) x*n*pc + kz0 + c;
  if(blockIdx.x + la < gridDim.x) {
    // tile T's 1024 rows: one 64-byte segment each, inside one line
    const unsigned T = blockIdx.x + la;
    const float2* h = a + (size_t)(T / tiles_z)*n*pc + (T % tiles_z)*RD_W;
#pragma unroll
    for(int q = 0; q < n/RD_NT; q++) prefetch_l2(h + (size_t)(threadIdx.x + RD_NT*q)*pc);
  }
  float2 v[32];
#pragma unroll
  for(int m = 0; m < 32; m++) v[m] = g[(size_t)(s + 32*m)*pc];
  rd_step_a<false>(v, c, s, sm, tw);
  __syncthreads();
  rd_step_b<false>(v, c, s, sm);
#pragma unroll
  for(int k2 = 0; k2 < 32; k2++) g[(size_t)(s + 32*k2)*pc] = v[bitrev(k2, 5)];
}

// XX, n = 1024: one block per tile (ky, kz block): forward along x, then
// the inverse of G into cc (and delta(k) into dk_out if asked) and the
// inverse of H = k_x G into b.  After the forward transform thread (c, k1)
// holds X[k1 + 32 k2] for every k2, which is exactly the input of the
// inverse's first step (no transposition there).  While the G inverse uses
// the registers and the transposition buffer, X waits in tensor memory:
// 64 columns of the thread's lane, warps w and w + 4 sharing a lane quarter
// (128 columns per block).
constexpr int XXR_TCOLS = 128;

// NY: ky rows per x plane of the work meshes (RD_N; fewer only for
// fused_pass_probe's slab)
template<int NY>
__global__ void __launch_bounds__(RD_NT, 2)
k_xx_rd(const float2* __restrict__ a, float2* __restrict__ b,
        float2* __restrict__ cc, float2* __restrict__ dk_out, float f1,
        const float2* __restrict__ tw, float* __restrict__ fill,
        size_t fill_chunks) {
  constexpr int n = RD_N, pc = RD_PC;
  constexpr size_t rs = (size_t) NY*RD_PC;
  extern __shared__ float2 sm[];
  __shared__ uint32_t tmem_base;
  const int warp = threadIdx.x >> 5;
  if(warp == 0) tmem_alloc(&tmem_base, XXR_TCOLS);
  tmem_fence_before();
  __syncthreads();
  tmem_fence_after();
  const uint32_t tx = tmem_base + ((uint32_t)(32*(warp & 3)) << 16) +
                      (uint32_t)(64*(warp >> 2));
  const int tiles_z = pc/RD_W;
  const int ky = blockIdx.x / tiles_z, kz0 = (blockIdx.x % tiles_z)*RD_W;
  const size_t off = (size_t) ky*pc + kz0;
  const int c = threadIdx.x & 7, s = threadIdx.x >> 3;
  const float2* g = a + off + c;
  float2 v[32];
#pragma unroll
  for(int m = 0; m < 32; m++) v[m] = g[(size_t)(s + 32*m)*rs];
  rd_step_a<false, true>(v, c, s, sm, tw);
  __syncthreads();
  rd_step_b<false, true>(v, c, s, sm);         // X[s + 32 k2] = v[bitrev(k2)]
  if(dk_out) {
    float2* d = dk_out + off + c;
#pragma unroll
    for(int k2 = 0; k2 < 32; k2++) d[(size_t)(s + 32*k2)*rs] = v[bitrev(k2, 5)];
  }
  {
    float st[64];
#pragma unroll
    for(int k2 = 0; k2 < 32; k2++) {
      st[2*k2] = v[bitrev(k2, 5)].x;
      st[2*k2 + 1] = v[bitrev(k2, 5)].y;
    }
    tmem_st64(tx, st);
  }
  // Green's function at (kx = s + 32 k2, ky, kz0 + c); u[k2] natural order.
  // One sweep over X forms G into u and H = k_x G back into X's
  // tensor-memory columns, so the H transform reads it without
  // evaluating the Green's function again.
  const int kz = kz0 + c;
  const float fy = (float)(ky <= n/2 ? ky : ky - n);
  const float fz = (float) kz;
  float2 u[32];
#pragma unroll
  for(int ch = 0; ch < 4; ch++) {
    uint32_t r[16];
    tmem_ld16(tx + 16*ch, r);
#pragma unroll
    for(int t = 0; t < 8; t++) {
      const int k2 = 8*ch + t;
      const int kx = s + 32*k2;
      const float fx = (float)(kx <= n/2 ? kx : kx - n);
      const float ksq = fx*fx + fy*fy + fz*fz;
      const float2 d = make_float2(__uint_as_float(r[2*t]),
                                   __uint_as_float(r[2*t + 1]));
      float2 g2 = make_float2(0.f, 0.f), h2 = make_float2(0.f, 0.f);
      if(!(ksq == 0.0f || kz > n/2)) {
        const float gg = f1/ksq;
        const float qh = gg*fx;
        g2 = make_float2(-gg*d.y, gg*d.x);
        h2 = make_float2(-qh*d.y, qh*d.x);
      }
      u[k2] = g2;
      r[2*t] = __float_as_uint(h2.x);
      r[2*t + 1] = __float_as_uint(h2.y);
    }
    tmem_st16(tx + 16*ch, r);
  }
#pragma unroll 1
  for(int is_h = 0; is_h < 2; is_h++) {
    if(is_h) {
#pragma unroll
      for(int ch = 0; ch < 4; ch++) {
        uint32_t r[16];
        tmem_ld16(tx + 16*ch, r);
#pragma unroll
        for(int t = 0; t < 8; t++)
          u[8*ch + t] = make_float2(__uint_as_float(r[2*t]), __uint_as_float(r[2*t + 1]));
      }
    }
    // inverse: step A over k2 in registers (thread s plays k1 of the
    // inverse decomposition), W_L^{-s n1}, transposition, step B over k1
    __syncthreads();                     // earlier reads of sm are done
    rd_step_a<true, true>(u, c, s, sm, tw);
    __syncthreads();
    rd_step_b<true, true>(u, c, s, sm);
    float2* o = (is_h ? b : cc) + off + c;
#pragma unroll
    for(int n2 = 0; n2 < 32; n2++) o[(size_t)(s + 32*n2)*rs] = u[bitrev(n2, 5)];
  }
  if(fill) {
    // FZ has consumed the density mesh: reset this block's share of it to
    // -1 (what the next deposit starts from) in 32-byte stores.  XX leaves
    // most of HBM's bandwidth unused, so this hides the clear's 4.3 GB.
    const size_t per = (fill_chunks + gridDim.x - 1)/gridDim.x;
    const size_t q0 = (size_t) blockIdx.x*per;
    const size_t q1 = q0 + per < fill_chunks ? q0 + per : fill_chunks;
    const float4 m1 = make_float4(-1.f, -1.f, -1.f, -1.f);
    for(size_t q = q0 + threadIdx.x; q < q1; q += RD_NT)
      st_global_v8(reinterpret_cast<float4*>(fill) + 2*q, m1, m1);
  }
  tmem_fence_before();
  __syncthreads();
  if(warp == 0) {
    tmem_fence_after();
    tmem_dealloc(tmem_base, XXR_TCOLS);
  }
}

// IY, n = 1024: three blocks per tile (x, kz block): 3t: a = IFy[c];
// 3t+1: d = IFy[k_y c]; 3t+2: b = IFy[b] (in place; no other block reads b).
__global__ void __launch_bounds__(RD_NT, 2)
k_iy_rd(float2* __restrict__ a, float2* __restrict__ b,
        const float2* __restrict__ cc, float2* __restrict__ d,
        const float2* __restrict__ tw, unsigned la) {
  constexpr int n = RD_N, pc = RD_PC;
  extern __shared__ float2 sm[];
  const int tiles_z = pc/RD_W;
  const int tile = blockIdx.x / 3, type = blockIdx.x % 3;
  const int x = tile / tiles_z, kz0 = (tile % tiles_z)*RD_W;
  const size_t off = (size_t) x*n*pc + kz0;
  const int c = threadIdx.x & 7, s = threadIdx.x >> 3;
  const float2* g = (type == 2 ? b : cc) + off + c;
  const unsigned T = blockIdx.x + la;
  if(T < gridDim.x && T % 3 != 1) {         // kinds 0 and 1 read the same tile
    const unsigned tt = T / 3;
    const float2* h = (T % 3 == 2 ? b : cc) + (size_t)(tt / tiles_z)*n*pc +
                      (tt % tiles_z)*RD_W;
#pragma unroll
    for(int q = 0; q < n/RD_NT; q++) prefetch_l2(h + (size_t)(threadIdx.x + RD_NT*q)*pc);
  }
  float2 v[32];
#pragma unroll
  for(int m = 0; m < 32; m++) v[m] = g[(size_t)(s + 32*m)*pc];
  if(type == 1) {
#pragma unroll
    for(int m = 0; m < 32; m++) {
      const int ky = s + 32*m;
      const float fy = (float)(ky <= n/2 ? ky : ky - n);
      v[m] = make_float2(fy*v[m].x, fy*v[m].y);
    }
  }
  rd_step_a<true>(v, c, s, sm, tw);
  __syncthreads();
  rd_step_b<true>(v, c, s, sm);
  float2* o = (type == 0 ? a : (type == 1 ? d : b)) + off + c;
#pragma unroll
  for(int k2 = 0; k2 < 32; k2++) o[(size_t)(s + 32*k2)*pc] = v[bitrev(k2, 5)];
}

// component `comp` of cells 2j and 2j+1 of a float4 row: (v.x, v.y); the z
// component also writes the fourth lane (0), so that every sector of the
// row is written whole
__device__ __forceinline__ void put_pair(float4* __restrict__ row, int j,
                                         int comp, float2 v) {
  float* c0 = reinterpret_cast<float*>(row + 2*j) + comp;
  float* c1 = reinterpret_cast<float*>(row + 2*j + 1) + comp;
  if(comp == 2) {
    *reinterpret_cast<float2*>(c0) = make_float2(v.x, 0.f);
    *reinterpret_cast<float2*>(c1) = make_float2(v.y, 0.f);
  }
  else { *c0 = v.x; *c1 = v.y; }
}

// --------------------------------------------------------------------
// IZ: C2R along z of three rows; f_z's row is multiplied by k_z first.
// The imaginary parts of the kz = 0 and kz = n/2 bins are dropped.
// Z_k = (X_k + conj X_{L-k}) + i w^k (X_k - conj X_{L-k}), w = e^{+2 pi i/n},
// z = inverse DFT_L(Z), out[2j] = Re z_j, out[2j+1] = Im z_j.
// --------------------------------------------------------------------
template<int R>
__global__ void __launch_bounds__(32*ROW_WARPS)
k_iz(const float2* __restrict__ a, const float2* __restrict__ b,
     const float2* __restrict__ c, float4* __restrict__ f4, int n, int pc,
     const float2* __restrict__ tw) {
  constexpr int L = 32*R, B = 32/R, SEQ = L + L/32 + 2;
  __shared__ float2 sm[ROW_WARPS][B*SEQ];
  const int warp = threadIdx.x >> 5, l = threadIdx.x & 31;
  const size_t row0 = ((size_t) blockIdx.x*ROW_WARPS + warp)*B;
  if(row0 >= (size_t) n*n) return;
  float2* base = sm[warp];
#pragma unroll 1
  for(int s = 0; s < 3; s++) {
    const float2* srcb = s == 0 ? b : (s == 1 ? c : a);
#pragma unroll 1
    for(int sq = 0; sq < B; sq++) {
      const float2* src = srcb + (row0 + sq)*pc;
      float2* col = base + sq*SEQ;
      for(int k = l; k < L; k += 32) {
        float2 xk = src[k];
        float2 xm = src[L - k];
        if(s == 2) {
          const float fk = (float) k, fm = (float)(L - k);
          xk = make_float2(fk*xk.x, fk*xk.y);
          xm = make_float2(fm*xm.x, fm*xm.y);
        }
        if(k == 0) { xk.y = 0.f; xm.y = 0.f; }       // DC and Nyquist: real part
        const float2 xc = cconj(xm);
        const float2 sum = cadd(xk, xc), dif_ = csub(xk, xc);
        const float2 w = k == 0 ? make_float2(1.f, 0.f) : cconj(__ldg(tw + k));
        const float2 wd = cmul(w, dif_);                // e^{+2 pi i k/n} d
        col[pidx(k)] = make_float2(sum.x - wd.y, sum.y + wd.x);   // + i w d
      }
    }
    __syncwarp();
    warp_fft_multi<R, true>(base, SEQ, Tw{tw, 2});
#pragma unroll 1
    for(int sq = 0; sq < B; sq++) {
      float4* dst = f4 + (row0 + sq)*n;
      const float2* col = base + sq*SEQ;
      for(int j = l; j < L; j += 32) put_pair(dst, j, s, col[pidx(j)]);
    }
    __syncwarp();
  }
}

// --------------------------------------------------------------------
// Register-direct IZ for n = 1024 (L = 512 = 32 x 16).  A warp takes two
// rows and their three components: lane l loads X[k] and X[L-k] for
// k = l + 32 m (m < 16) straight from HBM (both coalesced, the partner in
// reverse order), forms Z[k] and runs step A (16-point DFT over m, twiddle
// W_L^{l k1}) in registers for each row in turn; one transposition
// Y[q][l][k1] (row stride 17 words: conflict-free) hands each lane
// (q = l / 16, k1 = l % 16) its 32 inputs of step B, after which lane
// (q, k1) holds z[k1 + 16 k2], i.e. the real outputs of cells
// 2(k1 + 16 k2) and 2(k1 + 16 k2) + 1.  f_x and f_y wait in the lane's own
// tensor-memory columns (64 each) until f_z is done; then each lane writes
// its two adjacent cells in one 256-bit store.  Shared memory holds only the
// transposition,
// so four blocks (16 warps) share an SM.  Same arithmetic as k_iz (bitwise).
// --------------------------------------------------------------------
constexpr int IZR_WARPS = 4, IZR_SL = 17, IZR_SQ = 32*IZR_SL;
constexpr int IZR_TCOLS = 128;   // tensor-memory columns per block

__global__ void __launch_bounds__(32*IZR_WARPS, 4)
k_iz_rd(const float2* __restrict__ a, const float2* __restrict__ b,
        const float2* __restrict__ c, float4* __restrict__ f4,
        const float2* __restrict__ tw) {
  constexpr int n = RD_N, L = n/2, pc = RD_PC;
  __shared__ float2 sm[IZR_WARPS][2*IZR_SQ];
  __shared__ uint32_t tmem_base;
  const int warp = threadIdx.x >> 5, l = threadIdx.x & 31;
  if(warp == 0) tmem_alloc(&tmem_base, IZR_TCOLS);
  tmem_fence_before();
  __syncthreads();
  tmem_fence_after();
  // this warp's lane quarter; the grid covers the n^2 rows exactly
  const uint32_t tq = tmem_base + ((uint32_t)(32*warp) << 16);
  const size_t row0 = ((size_t) blockIdx.x*IZR_WARPS + warp)*2;
  float2* buf = sm[warp];
  const int q = l >> 4, k1b = l & 15;
#pragma unroll 1
  for(int src_i = 0; src_i < 3; src_i++) {
    const float2* srcb = src_i == 0 ? b : (src_i == 1 ? c : a);
#pragma unroll 1
    for(int r = 0; r < 2; r++) {
      const float2* src = srcb + (row0 + r)*pc;
      float2 xk[16], xm[16];
#pragma unroll
      for(int m = 0; m < 16; m++) {
        xk[m] = src[l + 32*m];
        xm[m] = src[L - l - 32*m];
      }
      float2 v[16];
#pragma unroll
      for(int m = 0; m < 16; m++) {
        const int k = l + 32*m;
        float2 x0 = xk[m], x1 = xm[m];
        if(src_i == 2) {
          const float fk = (float) k, fm = (float)(L - k);
          x0 = make_float2(fk*x0.x, fk*x0.y);
          x1 = make_float2(fm*x1.x, fm*x1.y);
        }
        if(k == 0) { x0.y = 0.f; x1.y = 0.f; }       // DC and Nyquist: real part
        const float2 xc = cconj(x1);
        const float2 sum = cadd(x0, xc), dif_ = csub(x0, xc);
        const float2 w = k == 0 ? make_float2(1.f, 0.f) : cconj(__ldg(tw + k));
        const float2 wd = cmul(w, dif_);
        v[m] = make_float2(sum.x - wd.y, sum.y + wd.x);
      }
      dif<16, true>(v);
#pragma unroll
      for(int k1 = 0; k1 < 16; k1++) {
        float2 y = v[bitrev(k1, 4)];
        if(k1 > 0 && l > 0) y = cmul(y, tw_dir<true>(__ldg(tw + 2*l*k1)));
        buf[r*IZR_SQ + l*IZR_SL + k1] = y;
      }
    }
    __syncwarp();
    float2 w[32];
#pragma unroll
    for(int j = 0; j < 32; j++) w[j] = buf[q*IZR_SQ + j*IZR_SL + k1b];
    __syncwarp();
    dif<32, true>(w);
    if(src_i < 2) {
      float st[64];
#pragma unroll
      for(int k2 = 0; k2 < 32; k2++) {
        st[2*k2] = w[bitrev(k2, 5)].x;
        st[2*k2 + 1] = w[bitrev(k2, 5)].y;
      }
      tmem_st64(tq + 64*src_i, st);
    }
    else {
      float4* dst = f4 + (row0 + q)*n;
#pragma unroll
      for(int ch = 0; ch < 4; ch++) {
        uint32_t rx[16], ry[16];
        tmem_ld16(tq + 16*ch, rx);
        tmem_ld16(tq + 64 + 16*ch, ry);
#pragma unroll
        for(int t = 0; t < 8; t++) {
          const int k2 = 8*ch + t, jj = k1b + 16*k2;
          const float2 vz = w[bitrev(k2, 5)];
          st_global_v8(dst + 2*jj,
                       make_float4(__uint_as_float(rx[2*t]), __uint_as_float(ry[2*t]), vz.x, 0.f),
                       make_float4(__uint_as_float(rx[2*t + 1]), __uint_as_float(ry[2*t + 1]), vz.y, 0.f));
        }
      }
    }
  }
  tmem_fence_before();
  __syncthreads();
  if(warp == 0) {
    tmem_fence_after();
    tmem_dealloc(tmem_base, IZR_TCOLS);
  }
}

// --------------------------------------------------------------------
// Register-direct FZ for n = 1024 (L = 512 = 32 x 16), two rows per warp:
// lane l loads Z[l + 32 m] (m < 16, Z_j = (x_2j, x_2j+1)) of each row
// straight from HBM, runs step A (16-point DFT over m, twiddle W_L^{l k1})
// in registers, and one transposition Y[q][l][k1] hands lane (q, k1) its
// step-B inputs.  After step B lane (q, k1) holds Zhat[k1 + 16 k2] of row
// q; the split X_k = (Z_k + conj Z_{L-k})/2 - i W^k (Z_k - conj Z_{L-k})/2
// needs the partner bin L - k, so Zhat goes through the (then free)
// transposition buffer in natural order once.  Same arithmetic as k_fz.
// --------------------------------------------------------------------
__global__ void __launch_bounds__(32*IZR_WARPS)
k_fz_rd(const float* __restrict__ in, float2* __restrict__ out,
        const float2* __restrict__ tw) {
  constexpr int n = RD_N, L = n/2, pc = RD_PC, ncz = n + 2;
  __shared__ float2 sm[IZR_WARPS][2*IZR_SQ];
  const int warp = threadIdx.x >> 5, l = threadIdx.x & 31;
  const size_t row0 = ((size_t) blockIdx.x*IZR_WARPS + warp)*2;
  float2* buf = sm[warp];
  const int q = l >> 4, k1b = l & 15;
  // both rows' loads in flight at once
  float2 vv[2][16];
#pragma unroll
  for(int r = 0; r < 2; r++) {
    const float2* src = reinterpret_cast<const float2*>(in + (row0 + r)*ncz);
#pragma unroll
    for(int m = 0; m < 16; m++) vv[r][m] = src[l + 32*m];
  }
#pragma unroll
  for(int r = 0; r < 2; r++) {
    float2 (&v)[16] = vv[r];
    dif<16, false>(v);
#pragma unroll
    for(int k1 = 0; k1 < 16; k1++) {
      float2 y = v[bitrev(k1, 4)];
      if(k1 > 0 && l > 0) y = cmul(y, __ldg(tw + 2*l*k1));
      buf[r*IZR_SQ + l*IZR_SL + k1] = y;
    }
  }
  __syncwarp();
  float2 w[32];
#pragma unroll
  for(int j = 0; j < 32; j++) w[j] = buf[q*IZR_SQ + j*IZR_SL + k1b];
  __syncwarp();
  dif<32, false>(w);
  // Zhat of row q in natural order: element e at buf[q*IZR_SQ + e]
#pragma unroll
  for(int k2 = 0; k2 < 32; k2++) buf[q*IZR_SQ + k1b + 16*k2] = w[bitrev(k2, 5)];
  __syncwarp();
#pragma unroll 1
  for(int r = 0; r < 2; r++) {
    const float2* col = buf + r*IZR_SQ;
    float2* dst = out + (row0 + r)*pc;
    for(int k = l; k <= L; k += 32) {
      const float2 zk = col[k == L ? 0 : k];
      const float2 zc = cconj(col[k == 0 ? 0 : L - k]);
      const float2 e = make_float2(0.5f*(zk.x + zc.x), 0.5f*(zk.y + zc.y));
      const float2 d = make_float2(0.5f*(zk.x - zc.x), 0.5f*(zk.y - zc.y));
      const float2 wk = k == L ? make_float2(-1.f, 0.f) : __ldg(tw + k);
      const float2 wd = cmul(wk, d);
      dst[k] = make_float2(e.x + wd.y, e.y - wd.x);
    }
  }
}

template<int L, int W>
constexpr size_t tile_smem() { return (size_t) W*TileSm<L>::CP*sizeof(float2); }

template<int RN, int W>  // RN: R of the length-n transforms (n = 32 RN); W: tile width
void run_pass(cudaStream_t s, int pass, const FusedBufs& f) {
  constexpr int L = 32*RN;
  constexpr size_t smem = tile_smem<L, W>();
  static int attr_device = -1, attr_device_rd = -1, rd_sms = 148;
  int dev = 0;
  cudaGetDevice(&dev);
  if(attr_device != dev) {
    cudaFuncSetAttribute(k_fy<RN, W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
    cudaFuncSetAttribute(k_xx<RN, W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) (2*smem));
    cudaFuncSetAttribute(k_iy<RN, W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) (2*smem));
    attr_device = dev;
  }
  const int n = f.n, pc = f.pc;
  // FZ / IZ: ROW_WARPS warps per block, 32/R rows per warp (R = n/64 there)
  const int rows_per_block = ROW_WARPS*(32/(RN/2 >= 1 ? RN/2 : 1));
  const unsigned rows_blocks = (unsigned)(((size_t) n*n + rows_per_block - 1)/rows_per_block);
  const unsigned tiles = (unsigned)((size_t) n*(pc/W));
  if(RN == 32 && W == RD_W && n == RD_N && pc == RD_PC) {
    if(attr_device_rd != dev) {
      cudaFuncSetAttribute(k_fy_rd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) RD_SMEM);
      cudaFuncSetAttribute(k_xx_rd<RD_N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) RD_SMEM);
      cudaFuncSetAttribute(k_iy_rd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) RD_SMEM);
      cudaDeviceGetAttribute(&rd_sms, cudaDevAttrMultiProcessorCount, dev);
      attr_device_rd = dev;
    }
    switch(pass) {
      case 0: k_fz_rd<<<(unsigned)((size_t) n*n/(2*IZR_WARPS)), 32*IZR_WARPS, 0, s>>>(
                  f.delta, f.A, f.tw); return;
      case 1: k_fy_rd<<<tiles, RD_NT, RD_SMEM, s>>>(f.A, f.tw, (unsigned) rd_sms); return;
      case 4: k_iz_rd<<<(unsigned)((size_t) n*n/(2*IZR_WARPS)), 32*IZR_WARPS, 0, s>>>(
                  f.A, f.B, f.D, f.f4, f.tw); return;
      case 2: {
        // the density mesh, n x n x (n + 2) floats, in 32-byte chunks
        const bool fill = fused_fills_mesh(f);
        const size_t chunks = fill ? (size_t) n*n*(n + 2)/8 : 0;
        k_xx_rd<RD_N><<<tiles, RD_NT, RD_SMEM, s>>>(f.A, f.B, f.C, f.dk_out, f.f1, f.tw,
                                              fill ? f.fill_mesh : nullptr, chunks);
        return;
      }
      case 3: k_iy_rd<<<3*tiles, RD_NT, RD_SMEM, s>>>(f.A, f.B, f.C, f.D, f.tw, (unsigned) rd_sms); return;
      default: break;
    }
  }
  switch(pass) {
    case 0: k_fz<RN/2><<<rows_blocks, 32*ROW_WARPS, 0, s>>>(f.delta, f.A, n, pc, f.tw); break;
    case 1: k_fy<RN, W><<<tiles, 32*W, smem, s>>>(f.A, n, pc, f.tw); break;
    case 2: k_xx<RN, W><<<tiles, 64*W, 2*smem, s>>>(f.A, f.B, f.C, f.dk_out, n, pc, f.f1, f.tw); break;
    case 3: k_iy<RN, W><<<tiles, 64*W, 2*smem, s>>>(f.A, f.B, f.C, f.D, n, pc, f.tw); break;
    case 4: k_iz<RN/2><<<rows_blocks, 32*ROW_WARPS, 0, s>>>(f.A, f.B, f.D, f.f4, n, pc, f.tw); break;
  }
}

}  // namespace

int fused_pitch(int n) { return ((n/2 + 1) + TILE_W - 1)/TILE_W*TILE_W; }

bool fused_fills_mesh(const FusedBufs& f) {
  return f.fill_mesh && f.n == RD_N && f.pc == RD_PC && f.tile == RD_W &&
         (reinterpret_cast<uintptr_t>(f.fill_mesh) & 31) == 0;
}


bool fused_supported(int n) {
  return n >= 64 && n <= 1024 && (n & (n - 1)) == 0;
}

void fused_init_constants() {}

void fused_twiddles(int n, std::vector<float2>& out) {
  out.resize(n);
  for(int j = 0; j < n; j++) {
    const double t = -2.0*M_PI*(double) j/(double) n;
    out[j] = make_float2((float) std::cos(t), (float) std::sin(t));
  }
}

template<int W>
void launch_w(cudaStream_t s, int pass, const FusedBufs& f) {
  switch(f.n) {
    case 64:   run_pass<2, W>(s, pass, f); break;
    case 128:  run_pass<4, W>(s, pass, f); break;
    case 256:  run_pass<8, W>(s, pass, f); break;
    case 512:  run_pass<16, W>(s, pass, f); break;
    case 1024: run_pass<32, W>(s, pass, f); break;
    default: break;
  }
}

namespace {
// the XX slab's ky rows: 32 or 64 (the slab's `planes`)

__global__ void k_probe_fill(float* __restrict__ p, size_t n, unsigned seed) {
  for(size_t i = blockIdx.x*(size_t) blockDim.x + threadIdx.x; i < n;
      i += (size_t) gridDim.x*blockDim.x) {
    unsigned h = (unsigned)(i*2654435761u) ^ seed;
    h ^= h >> 13; h *= 0x5bd1e995u; h ^= h >> 15;
    p[i] = (float)(h & 0xffffff)*(1.0f/16777216.0f) - 0.5f;
  }
}
}  // namespace

float fused_pass_probe(int pass, int planes, int reps) {
  if(pass < 0 || pass > 4) throw Error{FS2G_ERR_VALUE, "pass must be 0..4 (FZ FY XX IY IZ)"};
  if(planes < 1 || planes > RD_N) throw Error{FS2G_ERR_VALUE, "planes must be 1..1024"};
  if(pass == 2 && planes != 32 && planes != 64)
    throw Error{FS2G_ERR_VALUE, "the XX slab has 32 or 64 ky rows: planes must be 32 or 64"};
  if(reps < 1) throw Error{FS2G_ERR_VALUE, "reps must be >= 1"};
  constexpr int n = RD_N, pc = RD_PC;
  const size_t ne = (size_t) planes*n*pc;            // complex per work mesh
  const size_t nd = (size_t) planes*n*(n + 2);       // density floats
  const size_t nf = (size_t) planes*n*n;             // force cells
  std::vector<void*> bufs;
  auto alloc = [&](size_t bytes) {
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes);
    if(e != cudaSuccess) {
      for(void* q : bufs) cudaFree(q);
      throw_cuda(e, "pass probe buffers", __FILE__, __LINE__);
    }
    bufs.push_back(p);
    return p;
  };
  float ms_total = 0.0f;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  try {
    float* delta = (float*) alloc(nd*sizeof(float));
    float2* A = (float2*) alloc(ne*sizeof(float2));
    float2* B = (float2*) alloc(ne*sizeof(float2));
    float2* C = (float2*) alloc(ne*sizeof(float2));
    float2* D = (float2*) alloc(ne*sizeof(float2));
    float4* f4 = (float4*) alloc(nf*sizeof(float4));
    std::vector<float2> twh;
    fused_twiddles(n, twh);
    float2* tw = (float2*) alloc(twh.size()*sizeof(float2));
    FS2G_CUDA(cudaMemcpy(tw, twh.data(), twh.size()*sizeof(float2), cudaMemcpyHostToDevice));
    k_probe_fill<<<1184, 256>>>(delta, nd, 1u);
    k_probe_fill<<<1184, 256>>>((float*) A, 2*ne, 2u);
    k_probe_fill<<<1184, 256>>>((float*) B, 2*ne, 3u);
    k_probe_fill<<<1184, 256>>>((float*) C, 2*ne, 4u);
    FS2G_CUDA(cudaGetLastError());
    int dev = 0, sms = 148;
    FS2G_CUDA(cudaGetDevice(&dev));
    FS2G_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    FS2G_CUDA(cudaFuncSetAttribute(k_fy_rd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) RD_SMEM));
    FS2G_CUDA(cudaFuncSetAttribute(k_xx_rd<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) RD_SMEM));
    FS2G_CUDA(cudaFuncSetAttribute(k_xx_rd<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) RD_SMEM));
    FS2G_CUDA(cudaFuncSetAttribute(k_iy_rd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) RD_SMEM));
    const unsigned tiles = (unsigned)(planes*(pc/RD_W));
    const unsigned rows_blocks = (unsigned)((size_t) planes*n/(2*IZR_WARPS));
    FS2G_CUDA(cudaEventCreate(&e0));
    FS2G_CUDA(cudaEventCreate(&e1));
    FS2G_CUDA(cudaDeviceSynchronize());
    FS2G_CUDA(cudaEventRecord(e0));
    for(int r = 0; r < reps; r++) {
      switch(pass) {
        case 0: k_fz_rd<<<rows_blocks, 32*IZR_WARPS>>>(delta, A, tw); break;
        case 1: k_fy_rd<<<tiles, RD_NT, RD_SMEM>>>(A, tw, (unsigned) sms); break;
        case 2:
          if(planes == 64)
            k_xx_rd<64><<<tiles, RD_NT, RD_SMEM>>>(A, B, C, nullptr, -1e-9f, tw,
                                                   nullptr, 0);
          else
            k_xx_rd<32><<<tiles, RD_NT, RD_SMEM>>>(A, B, C, nullptr, -1e-9f, tw,
                                                   nullptr, 0);
          break;
        case 3: k_iy_rd<<<3*tiles, RD_NT, RD_SMEM>>>(A, B, C, D, tw, (unsigned) sms); break;
        default: k_iz_rd<<<rows_blocks, 32*IZR_WARPS>>>(A, B, D, f4, tw); break;
      }
    }
    FS2G_CUDA(cudaEventRecord(e1));
    FS2G_CUDA(cudaEventSynchronize(e1));
    FS2G_CUDA(cudaGetLastError());
    FS2G_CUDA(cudaEventElapsedTime(&ms_total, e0, e1));
  }
  catch(...) {
    if(e0) cudaEventDestroy(e0);
    if(e1) cudaEventDestroy(e1);
    for(void* q : bufs) cudaFree(q);
    throw;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  for(void* q : bufs) cudaFree(q);
  return ms_total/reps;
}

void launch_fused_pass(cudaStream_t s, int pass, const FusedBufs& f) {
  if(!fused_supported(f.n))
    throw Error{FS2G_ERR_VALUE, "fused FFT pipeline needs n in {64..1024}, a power of two"};
  switch(f.tile) {
    case 4: launch_w<4>(s, pass, f); break;
    default: launch_w<8>(s, pass, f); break;
  }
  cudaError_t e = cudaGetLastError();
  if(e != cudaSuccess) throw_cuda(e, "fused Poisson pass", __FILE__, __LINE__);
}

}  // namespace fs2g
