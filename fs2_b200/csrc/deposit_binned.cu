// deposit_binned.cu -- the CIC density deposit, py/pm.cpp:57-139, as a
// binned, shared-memory-staged deposit that writes every mesh cell once.
//
// The mesh is cut into tiles (one of the shapes in kShapes, powers of two
// along each axis; the last tile along an axis holds what is left of n).
// A particle whose base cell (i0) lies in tile T adds weight to cells of T
// and, when i0 sits on T's upper face along an axis, to the neighbouring
// tile along that axis (the cell i1 = i0 + 1, periodic).  So each particle
// is listed in the bins of the 1..8 tiles it touches:
//
//   k_bin_count    one pass over the positions (folding them into the box
//                  when asked, as the reference's wrap does): per-tile
//                  counts, one atomic per run of equal tiles in a warp
//   exclusive scan counts -> bin cursors
//   k_bin_scatter  the particle indices into their bins (a cursor advance
//                  per entry; afterwards cursor[t] is the end of bin t)
//   k_bin_deposit  one block per tile: the tile's cells accumulate in
//                  shared memory (lanes that share a base cell combine
//                  their weights first), then every cell of the tile is
//                  written once as -1 + sum
//
// After a deposit of the same particles (the time loop), count and scan
// give way to one pass into bins sized from the previous counts, with an
// overflow list for what does not fit (k_bin_scatter<..., true>).
//
// The mesh is never read, so the deposit needs no clear beforehand and no
// read-modify-write of HBM; cells that no particle reaches are written -1.
//
// A batched context (several same-sized realisations, gridDim.y the member
// in the particle passes) numbers the tiles of member m after those of
// members 0 .. m-1, so one scan and one deposit launch cover every member.
//
// The per-particle CIC indices and weights are the reference's products.
// The accumulator is 64-bit fixed point: every weight is rounded to a
// multiple of 2^-S and the integer sums are exact, so the result does not
// depend on the order of the additions at all -- bitwise reproducible.  S
// is chosen per call so that the total mass (np * pm_factor^3) stays below
// 2^62 units and a single weight below 2^32 units (S = 28 for pm_factor
// 2); the rounding of each weight (at most 2^-S-1) is far below the float
// spacing of the final -1 + sum.  This is the deterministic mode
// (FS2G_DEPOSIT_DETERMINISTIC) and the allocation-free density.
#include <algorithm>
#include <cmath>
#include <cub/cub.cuh>
#include "internal.h"

namespace fs2g {
namespace {

constexpr int DTPB = 256;

struct Cic1 { int i0, i1; float w0, w1; };

// py/pm.cpp:85-115: X = x*dx_inv (Float), i0 = (int)X, w1 = X - i0,
// w0 = 1 - w1, i0 >= n -> 0, i1 = i0 + 1 wrapped; i0 < 0 is flagged
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
  return __fmul_rn(__fmul_rn(__fmul_rn(a, b), c), d);   // fac*wx*wy*wz
}

__device__ __forceinline__ void flag(int* err, int code, long long detail) {
  if(atomicCAS(err, 0, code) == 0) err[1] = (int) detail;
}

// The tiles a particle touches: its base tile t0, and along each axis the
// step to the tile of i1 (d*, 0 when i1 lies in the same tile).  faces has
// bit 2 (x), 1 (y), 0 (z) set where that step leaves the tile; the other
// tiles are t0 + bx dx + by dy + bz dz for the non-empty subsets
// (bx << 2 | by << 1 | bz) of faces -- none for most particles.
struct TileSet {
  int t0, dx, dy, dz;
  unsigned faces;
  __device__ __forceinline__ int at(unsigned c) const {
    return t0 + ((c >> 2) & 1)*dx + ((c >> 1) & 1)*dy + (c & 1)*dz;
  }
};

// Tile sides are powers of two, given as shifts SX, SY, SZ (template
// arguments of the kernels below); the shapes built are listed in
// kShapes, and the result does not depend on the shape (integer sums).

// the tiles a particle touches: along each axis its base tile, plus the
// tile of i1 when that differs (i0 on the tile's upper face, or the
// periodic wrap of the last cell)
template<int SX, int SY, int SZ>
__device__ __forceinline__ TileSet tiles_of(const Cic1& cx, const Cic1& cy,
                                            const Cic1& cz, const BinGeom& g,
                                            int tile0) {
  const int ax0 = cx.i0 >> SX, ax1 = cx.i1 >> SX;
  const int ay0 = cy.i0 >> SY, ay1 = cy.i1 >> SY;
  const int az0 = cz.i0 >> SZ, az1 = cz.i1 >> SZ;
  TileSet s;
  s.t0 = tile0 + (ax0*g.nty + ay0)*g.ntz + az0;
  s.dx = (ax1 - ax0)*g.nty*g.ntz;
  s.dy = (ay1 - ay0)*g.ntz;
  s.dz = az1 - az0;
  s.faces = (ax1 != ax0 ? 4u : 0u) | (ay1 != ay0 ? 2u : 0u) | (az1 != az0 ? 1u : 0u);
  return s;
}

// Lanes of a warp whose keys are equal and adjacent form a run (particles
// in Lagrangian order fall into the same tile in runs).  Returns the run's
// first lane for this lane, and sets len (valid in the run's first lane).
// Dead lanes carry key -1 and form runs of their own.
__device__ __forceinline__ int run_head(int key, int lane, int& len) {
  const int prev = __shfl_up_sync(0xffffffffu, key, 1);
  const bool head = lane == 0 || key != prev;
  const unsigned heads = __ballot_sync(0xffffffffu, head);
  const unsigned later = heads & ~((2u << lane) - 1u);
  len = (later ? __ffs(later) - 1 : 32) - lane;
  return 31 - __clz(heads & ((2u << lane) - 1u));
}

// The counting pass takes PPT particles per thread, the j-th at block
// offset j*DTPB + threadIdx.x: all of a thread's position loads are issued
// before any is used (one particle per thread left the pass waiting on
// memory latency with 12 bytes in flight per thread).
constexpr int PPT = 4;

// the periodic fold of py/util.h:14-24 (single fold)
__device__ __forceinline__ float fold(float v, float L) {
  if(v < 0) v = __fadd_rn(v, L);
  if(v >= L) v = __fsub_rn(v, L);
  return v;
}

template<int SX, int SY, int SZ>
__global__ void __launch_bounds__(DTPB)
k_bin_count(float* __restrict__ x0, float* __restrict__ x1,
            float* __restrict__ x2, size_t np, float dx_inv, float L,
            int wrap, BinGeom g, uint32_t* __restrict__ counts,
            int* __restrict__ err) {
  // np: particles per member; member blockIdx.y
  const int lane = threadIdx.x & 31;
  const size_t b0 = (size_t) blockIdx.x*(DTPB*PPT) + threadIdx.x;
  const size_t m0 = blockIdx.y*np;
  const int tile0 = (int) blockIdx.y*g.ntx*g.nty*g.ntz;
  float xr[PPT][3];
#pragma unroll
  for(int j = 0; j < PPT; j++) {
    const size_t i = m0 + b0 + (size_t) j*DTPB;
    if(b0 + (size_t) j*DTPB < np) {
      xr[j][0] = x0[i]; xr[j][1] = x1[i]; xr[j][2] = x2[i];
    }
  }
#pragma unroll
  for(int j = 0; j < PPT; j++) {
    const size_t i = m0 + b0 + (size_t) j*DTPB;
    bool live = b0 + (size_t) j*DTPB < np;
    TileSet s{};
    if(live) {
      float v[3];
#pragma unroll
      for(int k = 0; k < 3; k++) {
        v[k] = wrap ? fold(xr[j][k], L) : xr[j][k];
        if(__float_as_uint(v[k]) != __float_as_uint(xr[j][k]))
          (k == 0 ? x0 : (k == 1 ? x1 : x2))[i] = v[k];
      }
      bool bad = false;
      const Cic1 cx = cic1(v[0], dx_inv, g.n, bad);
      const Cic1 cy = cic1(v[1], dx_inv, g.n, bad);
      const Cic1 cz = cic1(v[2], dx_inv, g.n, bad);
      if(bad) { flag(err, DEV_POSITION_OUT_OF_RANGE, (long long) i); live = false; }
      else s = tiles_of<SX, SY, SZ>(cx, cy, cz, g, tile0);
    }
    // base tile: one atomic per run of equal tiles in the warp
    const int t0 = live ? s.t0 : -1;
    int len;
    const int head = run_head(t0, lane, len);
    if(live && head == lane) atomicAdd(counts + t0, (uint32_t) len);
    // neighbouring tiles (about 1 particle in 6 at 16 x 16 x 32 tiles)
    if(live)
      for(unsigned c = s.faces; c; c = (c - 1) & s.faces)
        atomicAdd(counts + s.at(c), 1u);
  }
}

// The scatter takes PPT particles per thread like the count: all their
// position loads are issued first, then each particle's base-tile cursor
// advance (an atomic that returns the slot), so that a thread has PPT of
// those round trips to L2 in flight instead of one (one particle per
// thread left the pass waiting on them).
//
// FILL = false: the scatter of the two-pass binning (exact bins from the
// count and scan); with `only_if` given it does nothing unless *only_if is
// set (the fallback of the one-pass binning below).
// FILL = true: the one-pass binning.  Bins are laid out with room for the
// previous deposit's count plus a half plus 64 (bin_capacity), begin[t]
// their start; the pass folds and stores the positions (the count's job
// otherwise), claims slots, and stores an entry inside its bin's room or,
// beyond it, on an overflow list that is binned afterwards on its own
// (k_bin_counted, a scan, k_ovf_scatter).  Particles move far less than a
// tile per step, so few entries overflow; a full list sets *overflow, and
// the two-pass scatter then runs with the exact counts the claims produced.
__device__ __forceinline__ uint32_t bin_capacity(uint32_t c) {
  return c + (c >> 1) + 64u;
}

// an entry that found its bin's room full: onto the overflow list, whose
// entries are binned afterwards (k_ovf_scatter); a full list sets *overflow
__device__ __forceinline__ void spill(uint32_t* ovf_total, uint32_t* ovf_tile,
                                      uint32_t* ovf_idx, uint32_t ovf_cap,
                                      int* overflow, int t, uint32_t i) {
  const uint32_t o = atomicAdd(ovf_total, 1u);
  if(o < ovf_cap) { ovf_tile[o] = (uint32_t) t; ovf_idx[o] = i; }
  else *overflow = 1;
}

template<int SX, int SY, int SZ, bool FILL>
__global__ void __launch_bounds__(DTPB)
k_bin_scatter(float* __restrict__ x0, float* __restrict__ x1,
              float* __restrict__ x2, size_t np, float dx_inv, float L,
              int wrap, BinGeom g, uint32_t* __restrict__ cursor,
              uint32_t* __restrict__ idx, const uint32_t* __restrict__ begin,
              const uint32_t* __restrict__ prev, int* __restrict__ overflow,
              const int* __restrict__ only_if, int* __restrict__ err,
              uint32_t idx_cap, uint32_t* __restrict__ ovf_total,
              uint32_t* __restrict__ ovf_tile, uint32_t* __restrict__ ovf_idx,
              uint32_t ovf_cap) {
  if(!FILL && only_if && *only_if == 0) return;
  // np: particles per member; member blockIdx.y
  const int lane = threadIdx.x & 31;
  const size_t b0 = (size_t) blockIdx.x*(DTPB*PPT) + threadIdx.x;
  const size_t m0 = blockIdx.y*np;
  const int tile0 = (int) blockIdx.y*g.ntx*g.nty*g.ntz;
  float xr[PPT][3];
#pragma unroll
  for(int j = 0; j < PPT; j++) {
    const size_t i = m0 + b0 + (size_t) j*DTPB;
    if(b0 + (size_t) j*DTPB < np) {
      xr[j][0] = x0[i]; xr[j][1] = x1[i]; xr[j][2] = x2[i];
    }
  }
  bool live[PPT];
  int head[PPT], t0[PPT];
  uint32_t base[PPT];
  Cic1 cc[PPT][3];
#pragma unroll
  for(int j = 0; j < PPT; j++) {
    const size_t i = m0 + b0 + (size_t) j*DTPB;
    live[j] = b0 + (size_t) j*DTPB < np;
    t0[j] = -1;
    if(live[j]) {
      if(FILL && wrap) {
#pragma unroll
        for(int k = 0; k < 3; k++) {
          const float v = fold(xr[j][k], L);
          if(__float_as_uint(v) != __float_as_uint(xr[j][k]))
            (k == 0 ? x0 : (k == 1 ? x1 : x2))[i] = v;
          xr[j][k] = v;
        }
      }
      bool bad = false;
      cc[j][0] = cic1(xr[j][0], dx_inv, g.n, bad);
      cc[j][1] = cic1(xr[j][1], dx_inv, g.n, bad);
      cc[j][2] = cic1(xr[j][2], dx_inv, g.n, bad);
      if(bad) {
        if(FILL) flag(err, DEV_POSITION_OUT_OF_RANGE, (long long) i);
        live[j] = false;
      }
      else t0[j] = tile0 + ((cc[j][0].i0 >> SX)*g.nty + (cc[j][1].i0 >> SY))*g.ntz +
                   (cc[j][2].i0 >> SZ);
    }
    int len;
    head[j] = run_head(t0[j], lane, len);
    base[j] = 0;
    if(live[j] && head[j] == lane) base[j] = atomicAdd(cursor + t0[j], (uint32_t) len);
  }
#pragma unroll
  for(int j = 0; j < PPT; j++) {
    const uint32_t bj = __shfl_sync(0xffffffffu, base[j], head[j]);
    if(!live[j]) continue;
    const uint32_t i = (uint32_t)(m0 + b0 + (size_t) j*DTPB);
    const TileSet s = tiles_of<SX, SY, SZ>(cc[j][0], cc[j][1], cc[j][2], g, tile0);
    if(FILL) {
      uint32_t slot = bj + (lane - head[j]);
      // inside the bin's room (and the entry array: a layout too large for
      // it has set the flag already), else onto the overflow list
      if(slot < begin[t0[j]] + bin_capacity(prev[t0[j]]) && slot < idx_cap)
        idx[slot] = i;
      else spill(ovf_total, ovf_tile, ovf_idx, ovf_cap, overflow, t0[j], i);
      for(unsigned c = s.faces; c; c = (c - 1) & s.faces) {
        const int t = s.at(c);
        slot = atomicAdd(cursor + t, 1u);
        if(slot < begin[t] + bin_capacity(prev[t]) && slot < idx_cap) idx[slot] = i;
        else spill(ovf_total, ovf_tile, ovf_idx, ovf_cap, overflow, t, i);
      }
    }
    else {
      idx[bj + (lane - head[j])] = i;
      for(unsigned c = s.faces; c; c = (c - 1) & s.faces)
        idx[atomicAdd(cursor + s.at(c), 1u)] = i;
    }
  }
}

// one-pass binning, before the fill: begin[t] = room of bin t (from the
// previous deposit's counts in prev), to be scanned
__global__ void k_bin_rooms(const uint32_t* __restrict__ prev,
                            uint32_t* __restrict__ room, int ntiles) {
  for(int t = blockIdx.x*blockDim.x + threadIdx.x; t < ntiles;
      t += gridDim.x*blockDim.x)
    room[t] = bin_capacity(prev[t]);
}

// after the scan of the rooms into cursor: begin[t] = cursor[t]; the
// layout must fit the entry array (else *flag, the two-pass fallback)
__global__ void k_bin_plan(const uint32_t* __restrict__ cursor,
                           uint32_t* __restrict__ begin,
                           const uint32_t* __restrict__ prev, int ntiles,
                           size_t cap, int* __restrict__ flag) {
  for(int t = blockIdx.x*blockDim.x + threadIdx.x; t < ntiles;
      t += gridDim.x*blockDim.x) {
    begin[t] = cursor[t];
    if(t == ntiles - 1 && (size_t) cursor[t] + bin_capacity(prev[t]) > cap)
      *flag = 1;
  }
}

// after the fill: the exact counts (claims, whether stored or not) into
// counts (which held the previous deposit's), the entries stored in the
// bin into len, cursor moved back to the end of those, and the overflow
// list's share of the bin into olen
__global__ void k_bin_counted(uint32_t* __restrict__ cursor,
                              const uint32_t* __restrict__ begin,
                              uint32_t* __restrict__ counts,
                              uint32_t* __restrict__ len,
                              uint32_t* __restrict__ olen, int ntiles) {
  for(int t = blockIdx.x*blockDim.x + threadIdx.x; t < ntiles;
      t += gridDim.x*blockDim.x) {
    const uint32_t room = bin_capacity(counts[t]);
    const uint32_t c = cursor[t] - begin[t];
    const uint32_t stored = c < room ? c : room;
    counts[t] = c;
    len[t] = stored;
    olen[t] = c - stored;
    cursor[t] = begin[t] + stored;
  }
}

// the overflow list into per-bin segments: entry o of bin t goes to
// ostart[t] + (its rank among bin t's, by an atomic on ocur[t])
__global__ void k_ovf_scatter(const uint32_t* __restrict__ ovf_total,
                              const uint32_t* __restrict__ ovf_tile,
                              const uint32_t* __restrict__ ovf_idx,
                              uint32_t ovf_cap,
                              const uint32_t* __restrict__ ostart,
                              uint32_t* __restrict__ ocur,
                              uint32_t* __restrict__ ovf_sorted,
                              const int* __restrict__ flag) {
  if(*flag) return;                 // the full fallback takes over
  const uint32_t m = min(*ovf_total, ovf_cap);
  for(uint32_t o = blockIdx.x*blockDim.x + threadIdx.x; o < m;
      o += gridDim.x*blockDim.x) {
    const uint32_t t = ovf_tile[o];
    ovf_sorted[ostart[t] + atomicAdd(ocur + t, 1u)] = ovf_idx[o];
  }
}

// the full fallback, after its scatter: every entry is in its bin
__global__ void k_bin_fixlen(const int* __restrict__ flag,
                             const uint32_t* __restrict__ counts,
                             uint32_t* __restrict__ len, int ntiles) {
  if(*flag == 0) return;
  for(int t = blockIdx.x*blockDim.x + threadIdx.x; t < ntiles;
      t += gridDim.x*blockDim.x)
    len[t] = counts[t];
}

// the fallback's cursors: the exact layout's starts, if the fill overflowed
__global__ void k_bin_rewind(const int* __restrict__ flag,
                             const uint32_t* __restrict__ start,
                             uint32_t* __restrict__ cursor, int ntiles) {
  if(*flag == 0) return;
  for(int t = blockIdx.x*blockDim.x + threadIdx.x; t < ntiles;
      t += gridDim.x*blockDim.x)
    cursor[t] = start[t];
}

// The 64-bit fixed-point accumulator, two's complement (a weight below 0 --
// a position in (-1, 0) cell, which the reference's truncation maps to
// cell 0 with w1 < 0 -- adds modulo 2^64 and the signed reading of the sum
// is exact), held as two 32-bit words per cell, lo and hi.  Shared-memory
// 64-bit adds are compare-and-swap loops on this GPU, 32-bit integer adds
// are native: a weight v adds its low word to lo with one native add that
// returns the old value, which tells whether the word wrapped, and hi
// receives v's high word plus that carry -- nothing at all in the common
// case, since the scale keeps every single weight below 2^32 (the shift S
// is at most 31 - ceil(log2 pm_factor^3)).  hi * 2^32 + lo is the exact sum
// modulo 2^64.  (Three 16/16/32-bit limbs with carry-free native adds
// measured slower: three adds per corner and 12 bytes per cell.)
template<int SX, int SY, int SZ>
__host__ __device__ constexpr size_t deposit_smem() {
  return ((size_t) 1 << (SX + SY + SZ))*8;
}

typedef unsigned long long u64;

__device__ __forceinline__ u64 to_fixed(float w, float scale) {
  return (u64) __float2ll_rn(__fmul_rn(w, scale));   // exact scaling by 2^S
}

// six 256-thread blocks per SM (at most 42 registers), the shared-memory
// carveout at its maximum so that the accumulators of six blocks fit
template<int SX, int SY, int SZ>
__global__ void __launch_bounds__(DTPB, 6)
k_bin_deposit(const float* __restrict__ x0, const float* __restrict__ x1,
              const float* __restrict__ x2, const uint32_t* __restrict__ idx,
              const uint32_t* __restrict__ bin_end,
              const uint32_t* __restrict__ bin_len,
              const uint32_t* __restrict__ ovf_sorted,
              const uint32_t* __restrict__ ovf_start,
              const uint32_t* __restrict__ counts, float* __restrict__ mesh,
              float dx_inv, float fac, BinGeom g, float scale,
              double inv_scale) {
  // bin t's entries: bin_len[t] in idx ending at bin_end[t], then (one-pass
  // binning, ovf_sorted given) counts[t] - bin_len[t] more in ovf_sorted
  // from ovf_start[t]
  constexpr int TX = 1 << SX, TY = 1 << SY, TZ = 1 << SZ;
  constexpr int NCELLS = TX*TY*TZ;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint32_t* acc_lo = reinterpret_cast<uint32_t*>(smem_raw);
  uint32_t* acc_hi = acc_lo + NCELLS;
  const int n = g.n;
  const size_t ncz = 2*(size_t)(n/2 + 1);
  const int lane = threadIdx.x & 31;
  const int t = blockIdx.x;                 // member t / ntiles
  const int ntiles = g.ntx*g.nty*g.ntz;
  const int tl = t % ntiles;
  mesh += (size_t)(t/ntiles)*((size_t) n*n*ncz);
  const int tz = tl % g.ntz, ty = (tl/g.ntz) % g.nty, tx = tl/(g.ntz*g.nty);
  const int ox = tx << SX, oy = ty << SY, oz = tz << SZ;
  const uint32_t nb = bin_len[t], begin = bin_end[t] - nb;
  const uint32_t no = ovf_sorted ? counts[t] - nb : 0u;
  const uint32_t obegin = ovf_sorted ? ovf_start[t] : 0u;
  const uint32_t total = nb + no;
  auto entry = [&](uint32_t e) {
    return e < nb ? idx[begin + e] : ovf_sorted[obegin + (e - nb)];
  };
  {
    uint4* z = reinterpret_cast<uint4*>(smem_raw);
    for(int c = threadIdx.x; c < (int)(deposit_smem<SX, SY, SZ>()/16); c += blockDim.x)
      z[c] = make_uint4(0, 0, 0, 0);
  }
  __syncthreads();
  // block-uniform loop: every lane of every warp takes part in the
  // warp-wide votes below.  The next round's bin entry is loaded while
  // this round's positions are, so each round waits on one global load.
  uint32_t inext = threadIdx.x < total ? entry(threadIdx.x) : 0u;
  for(uint32_t e0 = 0; e0 < total; e0 += blockDim.x) {
    const uint32_t e = e0 + threadIdx.x;
    const bool live = e < total;
    const uint32_t i = inext;
    if(e + blockDim.x < total) inext = entry(e + blockDim.x);
    Cic1 cx{0, 0, 0.f, 0.f}, cy = cx, cz = cx;
    if(live) {
      bool bad = false;
      cx = cic1(x0[i], dx_inv, n, bad);
      cy = cic1(x1[i], dx_inv, n, bad);
      cz = cic1(x2[i], dx_inv, n, bad);
    }
    u64 w[8];
    w[0] = to_fixed(w3(fac, cx.w0, cy.w0, cz.w0), scale);
    w[1] = to_fixed(w3(fac, cx.w0, cy.w0, cz.w1), scale);
    w[2] = to_fixed(w3(fac, cx.w0, cy.w1, cz.w0), scale);
    w[3] = to_fixed(w3(fac, cx.w0, cy.w1, cz.w1), scale);
    w[4] = to_fixed(w3(fac, cx.w1, cy.w0, cz.w0), scale);
    w[5] = to_fixed(w3(fac, cx.w1, cy.w0, cz.w1), scale);
    w[6] = to_fixed(w3(fac, cx.w1, cy.w1, cz.w0), scale);
    w[7] = to_fixed(w3(fac, cx.w1, cy.w1, cz.w1), scale);
    // lanes with the same base cell add their weights into one lane
    const unsigned live_mask = __ballot_sync(0xffffffffu, live);
    if(live) {
      const unsigned long long key =
          ((unsigned long long) cx.i0*(unsigned) n + (unsigned) cy.i0)*
          (unsigned) n + (unsigned) cz.i0;
      const unsigned peers = __match_any_sync(live_mask, key);
      const int leader = __ffs(peers) - 1;
      bool mine = true;
      if(__popc(peers) > 1) {
        unsigned rest = peers & ~(1u << leader);
        while(rest) {
          const int src = __ffs(rest) - 1;
          rest &= rest - 1;
#pragma unroll
          for(int o = 0; o < 8; o++) {
            const u64 v = __shfl_sync(peers, w[o], src);
            if(lane == leader) w[o] += v;
          }
        }
        mine = lane == leader;
      }
      if(mine) {
        // the corners inside this tile (local coordinates)
        const int lx[2] = {cx.i0 - ox, cx.i1 - ox};
        const int ly[2] = {cy.i0 - oy, cy.i1 - oy};
        const int lz[2] = {cz.i0 - oz, cz.i1 - oz};
#pragma unroll
        for(int o = 0; o < 8; o++) {
          const int a = lx[(o >> 2) & 1], b = ly[(o >> 1) & 1], c = lz[o & 1];
          if((unsigned) a < (unsigned) TX && (unsigned) b < (unsigned) TY &&
             (unsigned) c < (unsigned) TZ) {
            const int cell = (a << (SY + SZ)) | (b << SZ) | c;
            const uint32_t vl = (uint32_t) w[o], vh = (uint32_t)(w[o] >> 32);
            const uint32_t old = atomicAdd(acc_lo + cell, vl);
            const uint32_t h = vh + (old + vl < old ? 1u : 0u);
            if(h) atomicAdd(acc_hi + cell, h);
          }
        }
      }
    }
  }
  __syncthreads();
  // every cell of the tile once: -1 + sum, rows of TZ cells along z
  const int ex = min(TX, n - ox), ey = min(TY, n - oy), ez = min(TZ, n - oz);
  float* base = mesh + ((size_t) ox*n + oy)*ncz + oz;
  for(int c = threadIdx.x; c < NCELLS; c += blockDim.x) {
    const int lz = c & (TZ - 1), ly = (c >> SZ) & (TY - 1), lx = c >> (SY + SZ);
    if(lx < ex && ly < ey && lz < ez)
      base[((size_t) lx*n + ly)*ncz + lz] = __double2float_rn(
          __dsub_rn(__dmul_rn((double)(long long)(((u64) acc_hi[c] << 32) | acc_lo[c]),
                              inv_scale), 1.0));
  }
}

// The tile shapes built (log2 of the sides x, y, z).  Shape 0 is the
// default and the allocation-free entry point's; the others trade tile
// count (bins, scan length, face duplicates) against shared memory per
// block (8 bytes a cell) and blocks per SM.
struct ShapeDesc { int sx, sy, sz; };
constexpr ShapeDesc kShapes[BIN_SHAPES] = {
    {4, 4, 5},     // 16 x 16 x 32, 64 KB
    {4, 3, 5},     // 16 x  8 x 32, 32 KB
    {3, 3, 5},     //  8 x  8 x 32, 16 KB
    {3, 3, 4},     //  8 x  8 x 16,  8 KB
    {2, 2, 5}};    //  4 x  4 x 32,  4 KB

template<int SX, int SY, int SZ>
cudaError_t run_shape(cudaStream_t stream, float* x0, float* x1, float* x2,
                      size_t np, float* mesh, const BinGeom& g, float dx_inv,
                      float fac, float boxsize, bool wrap,
                      const BinScratch& sc, int* err, int batch, bool reuse) {
  const int ntiles = g.ntx*g.nty*g.ntz*batch;         // every member's tiles
  const size_t npm = np/(size_t) batch;              // particles per member
  const unsigned tblocks = (unsigned) std::min(1024, (ntiles + 255)/256);
  cudaError_t e = cudaSuccess;
  if(np > 0 && reuse) {
    // one pass over the particles into bins sized from the previous
    // deposit's counts (sc.counts on entry); entries beyond a bin's room go
    // to the overflow list, binned afterwards on its own; the two-pass
    // scatter only if the list itself fills up
    const dim3 cblocks((unsigned)((npm + DTPB*PPT - 1)/(DTPB*PPT)),
                       (unsigned) batch);
    e = cudaMemsetAsync(sc.overflow, 0, sizeof(int), stream);
    if(e == cudaSuccess) e = cudaMemsetAsync(sc.ovf_total, 0, sizeof(uint32_t), stream);
    if(e == cudaSuccess) e = cudaMemsetAsync(sc.ocur, 0, (size_t) ntiles*4, stream);
    if(e != cudaSuccess) return e;
    k_bin_rooms<<<tblocks, 256, 0, stream>>>(sc.counts, sc.begin, ntiles);
    size_t tb = sc.temp_bytes;
    e = cub::DeviceScan::ExclusiveSum(sc.temp, tb, sc.begin, sc.cursor,
                                      ntiles, stream);
    if(e != cudaSuccess) return e;
    k_bin_plan<<<tblocks, 256, 0, stream>>>(sc.cursor, sc.begin, sc.counts,
                                            ntiles, sc.idx_cap, sc.overflow);
    k_bin_scatter<SX, SY, SZ, true><<<cblocks, DTPB, 0, stream>>>(
        x0, x1, x2, npm, dx_inv, boxsize, wrap ? 1 : 0, g, sc.cursor, sc.idx,
        sc.begin, sc.counts, sc.overflow, nullptr, err, (uint32_t) sc.idx_cap,
        sc.ovf_total, sc.ovf_tile, sc.ovf_idx, (uint32_t) sc.ovf_cap);
    k_bin_counted<<<tblocks, 256, 0, stream>>>(sc.cursor, sc.begin, sc.counts,
                                               sc.len, sc.olen, ntiles);
    tb = sc.temp_bytes;
    e = cub::DeviceScan::ExclusiveSum(sc.temp, tb, sc.olen, sc.ostart,
                                      ntiles, stream);
    if(e != cudaSuccess) return e;
    k_ovf_scatter<<<(unsigned) std::min<size_t>(1024, (sc.ovf_cap + 255)/256), 256, 0,
                    stream>>>(sc.ovf_total, sc.ovf_tile, sc.ovf_idx,
                              (uint32_t) sc.ovf_cap, sc.ostart, sc.ocur,
                              sc.ovf_sorted, sc.overflow);
    // the full fallback (does nothing unless *overflow)
    tb = sc.temp_bytes;
    e = cub::DeviceScan::ExclusiveSum(sc.temp, tb, sc.counts, sc.begin,
                                      ntiles, stream);
    if(e != cudaSuccess) return e;
    k_bin_rewind<<<tblocks, 256, 0, stream>>>(sc.overflow, sc.begin, sc.cursor,
                                              ntiles);
    k_bin_scatter<SX, SY, SZ, false><<<cblocks, DTPB, 0, stream>>>(
        x0, x1, x2, npm, dx_inv, boxsize, 0, g, sc.cursor, sc.idx, nullptr,
        nullptr, nullptr, sc.overflow, err, 0u, nullptr, nullptr, nullptr, 0u);
    k_bin_fixlen<<<tblocks, 256, 0, stream>>>(sc.overflow, sc.counts, sc.len,
                                              ntiles);
  }
  else if(np > 0) {
    e = cudaMemsetAsync(sc.counts, 0, (size_t) ntiles*4, stream);
    if(e != cudaSuccess) return e;
    const dim3 cblocks((unsigned)((npm + DTPB*PPT - 1)/(DTPB*PPT)),
                       (unsigned) batch);
    k_bin_count<SX, SY, SZ><<<cblocks, DTPB, 0, stream>>>(
        x0, x1, x2, npm, dx_inv, boxsize, wrap ? 1 : 0, g, sc.counts, err);
    size_t tb = sc.temp_bytes;
    e = cub::DeviceScan::ExclusiveSum(sc.temp, tb, sc.counts, sc.cursor,
                                      ntiles, stream);
    if(e != cudaSuccess) return e;
    k_bin_scatter<SX, SY, SZ, false><<<cblocks, DTPB, 0, stream>>>(
        x0, x1, x2, npm, dx_inv, boxsize, 0, g, sc.cursor, sc.idx, nullptr,
        nullptr, nullptr, nullptr, err, 0u, nullptr, nullptr, nullptr, 0u);
  }
  else {
    e = cudaMemsetAsync(sc.counts, 0, (size_t) ntiles*4, stream);
    if(e == cudaSuccess) e = cudaMemsetAsync(sc.cursor, 0, (size_t) ntiles*4, stream);
    if(e != cudaSuccess) return e;
  }
  // each member's mass bounds its cells: the same shift as a run alone
  // ... and keeps a single weight (at most pm_factor^3 for positions in
  // the box) below 2^32, so that the high word rarely changes
  const int S = std::min(fixed_point_shift(npm, fac),
                         std::max(16, 31 - (int) std::ceil(std::log2(
                             std::max(1.0f, std::fabs(fac))))));
  const float scale = std::ldexp(1.0f, S);
  const double inv_scale = std::ldexp(1.0, -S);
  // one block per tile: the block scheduler balances the uneven bins
  constexpr int cells = 1 << (SX + SY + SZ);
  constexpr int nt = cells >= 4*DTPB ? DTPB : cells/4;
  k_bin_deposit<SX, SY, SZ><<<(unsigned) ntiles, nt,
                              deposit_smem<SX, SY, SZ>(), stream>>>(
      x0, x1, x2, sc.idx, sc.cursor, (np > 0 && reuse) ? sc.len : sc.counts,
      (np > 0 && reuse) ? sc.ovf_sorted : nullptr, sc.ostart, sc.counts, mesh,
      dx_inv, fac, g, scale, inv_scale);
  return cudaGetLastError();
}

template<int SX, int SY, int SZ>
cudaError_t smem_limit() {
  cudaError_t e = cudaFuncSetAttribute(k_bin_deposit<SX, SY, SZ>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int) deposit_smem<SX, SY, SZ>());
  if(e == cudaSuccess)
    e = cudaFuncSetAttribute(k_bin_deposit<SX, SY, SZ>,
                             cudaFuncAttributePreferredSharedMemoryCarveout,
                             (int) cudaSharedmemCarveoutMaxShared);
  return e;
}

}  // namespace

BinGeom bin_geometry(int n, int shape) {
  if(shape < 0 || shape >= BIN_SHAPES) shape = 0;
  BinGeom g;
  g.n = n;
  g.shape = shape;
  g.tx = 1 << kShapes[shape].sx;
  g.ty = 1 << kShapes[shape].sy;
  g.tz = 1 << kShapes[shape].sz;
  g.ntx = (n + g.tx - 1)/g.tx; g.nty = (n + g.ty - 1)/g.ty;
  g.ntz = (n + g.tz - 1)/g.tz;
  return g;
}

size_t bin_scan_temp_bytes(int ntiles) {
  size_t b = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, b, (uint32_t*) nullptr,
                                (uint32_t*) nullptr, ntiles);
  return b;
}

int fixed_point_shift(size_t np, float fac) {
  // 2^S * np * fac < 2^62 (the sum of every weight -- a cell holding all
  // the mass -- still fits), S in [16, 40]
  const double mass = std::max(1.0, (double) np*(double) std::fabs(fac));
  int S = 62 - (int) std::ceil(std::log2(mass + 1.0));
  return std::max(16, std::min(40, S));
}

cudaError_t deposit_binned_on(cudaStream_t stream, float* x0, float* x1,
                              float* x2, size_t np, float* mesh, int n,
                              float dx_inv, float fac, float boxsize,
                              bool wrap, const BinScratch& sc, int* err,
                              int batch, int shape, bool reuse) {
  const BinGeom g = bin_geometry(n, shape);
  switch(g.shape) {
    case 1: return run_shape<4, 3, 5>(stream, x0, x1, x2, np, mesh, g, dx_inv, fac,
                                      boxsize, wrap, sc, err, batch, reuse);
    case 2: return run_shape<3, 3, 5>(stream, x0, x1, x2, np, mesh, g, dx_inv, fac,
                                      boxsize, wrap, sc, err, batch, reuse);
    case 3: return run_shape<3, 3, 4>(stream, x0, x1, x2, np, mesh, g, dx_inv, fac,
                                      boxsize, wrap, sc, err, batch, reuse);
    case 4: return run_shape<2, 2, 5>(stream, x0, x1, x2, np, mesh, g, dx_inv, fac,
                                      boxsize, wrap, sc, err, batch, reuse);
    default: return run_shape<4, 4, 5>(stream, x0, x1, x2, np, mesh, g, dx_inv, fac,
                                       boxsize, wrap, sc, err, batch, reuse);
  }
}

cudaError_t deposit_binned_set_smem_limits() {
  cudaError_t e = smem_limit<4, 4, 5>();
  if(e == cudaSuccess) e = smem_limit<4, 3, 5>();
  if(e == cudaSuccess) e = smem_limit<3, 3, 5>();
  if(e == cudaSuccess) e = smem_limit<3, 3, 4>();
  if(e == cudaSuccess) e = smem_limit<2, 2, 5>();
  return e;
}

}  // namespace fs2g
