// internal.h -- shared declarations of libfs2gpu (not part of the C ABI).
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>
#include <map>
#include <cuda_runtime.h>
#include <cufft.h>

#include "../../include/fs2gpu.h"

namespace fs2g {

// ---------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------
// A failing call stores its message here and returns a negative code.
void set_error(const std::string& msg);
int fail(int code, const std::string& msg);

struct Error {            // thrown inside the library, caught at the ABI
  int code;
  std::string msg;
};

[[noreturn]] void throw_cuda(cudaError_t e, const char* what, const char* file,
                             int line);

// run f, turning anything it throws into a status code (the ABI never throws)
template<class F> int guarded(F&& f) {
  try { f(); return FS2G_OK; }
  catch(const Error& e) { return fail(e.code, e.msg); }
  catch(const std::bad_alloc&) { return fail(FS2G_ERR_MEMORY, "out of host memory"); }
  catch(const std::exception& e) { return fail(FS2G_ERR_RUNTIME, e.what()); }
  catch(...) { return fail(FS2G_ERR_RUNTIME, "unknown error"); }
}
[[noreturn]] void throw_cufft(cufftResult r, const char* what,
                              const char* file, int line);

#define FS2G_CUDA(call) do { cudaError_t e_ = (call); \
  if(e_ != cudaSuccess) ::fs2g::throw_cuda(e_, #call, __FILE__, __LINE__); } while(0)
#define FS2G_CUFFT(call) do { cufftResult r_ = (call); \
  if(r_ != CUFFT_SUCCESS) ::fs2g::throw_cufft(r_, #call, __FILE__, __LINE__); } while(0)
#define FS2G_LAUNCHED(ctx) do { cudaError_t e_ = cudaGetLastError(); \
  if(e_ != cudaSuccess) ::fs2g::throw_cuda(e_, "kernel launch", __FILE__, __LINE__); \
  (ctx)->kernel_launches++; } while(0)

// device error word codes (ctx->d_err[0])
enum DeviceError : int {
  DEV_OK = 0,
  DEV_POSITION_OUT_OF_RANGE = 1,   // a cell index below 0 in deposit/gather
};

// ---------------------------------------------------------------------
// timing stages
// ---------------------------------------------------------------------
enum Stage : int {
  ST_WRAP = 0, ST_CLEAR, ST_DEPOSIT, ST_SORT, ST_R2C, ST_FORCE_K, ST_C2R,
  ST_GATHER, ST_KICK, ST_DRIFT, ST_KICK_DRIFT, ST_LPT_K, ST_LPT_FFT,
  ST_LPT_REAL, ST_LPT_PARTICLES, ST_COPY, ST_FZ, ST_FY, ST_XX, ST_IY, ST_IZ,
  ST_NSTAGES
};
extern const char* const stage_names[ST_NSTAGES];

// ---------------------------------------------------------------------
// FFT plans: in-place / out-of-place 3-D R2C and C2R on the padded real
// layout [n][n][2(n/2+1)] and the complex layout [n][n][n/2+1].
// ---------------------------------------------------------------------
enum PlanKind : int { PLAN_R2C_INPLACE = 0, PLAN_R2C_OUTOFPLACE,
                      PLAN_C2R_INPLACE };

struct FFTPlans {
  std::map<std::pair<int,int>, cufftHandle> plans;
  void* work = nullptr;
  size_t work_size = 0;
};

// ---------------------------------------------------------------------
// objects behind the opaque ABI handles
// ---------------------------------------------------------------------
struct StageEvent { int stage; cudaEvent_t start, stop; };

}  // namespace fs2g

struct fs2g_fft {
  fs2g_ctx* ctx;
  int nc;
  float* d_fx;        // padded real mesh [nc][nc][2(nc/2+1)]
  bool owned;         // false: the PM mesh of a context
};

struct fs2g_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;       // active stream
  cudaStream_t own_stream = nullptr;
  // second stream for host copies split in two (made on first use)
  cudaStream_t aux_stream = nullptr;
  cudaEvent_t aux_fork = nullptr, aux_join = nullptr;
  int* d_err = nullptr;                // device error word [0]=code [1]=detail
  long kernel_launches = 0;
  int sm_count = 148;
  // Realisations per PM mesh set: 1 for every public context; an
  // ensemble's size class runs its members as one batch (stacked meshes,
  // batched transforms, one particle set of batch x np particles, member m
  // owning [m np_m, (m+1) np_m)).  Fixed when the context is made.
  int batch = 1;

  // PM module state (py/pm.cpp:22-30)
  int pm_nc = 0;
  double pm_factor = 0.0;
  float pm_boxsize = 0.0f;
  int pm_status = FS2G_PM_DONE;
  int deposit_mode = FS2G_DEPOSIT_ATOMIC;
  int check = 0;
  float* mesh = nullptr;               // padded real mesh; after force: f_z
  float2* delta_k = nullptr;           // R2C output, [n][n][n/2+1]
  float* fmesh[2] = {nullptr, nullptr};  // f_x, f_y meshes (in-place C2R)
  // cuFFT path: where the force's three real meshes go, when set (the
  // differentiable run's per-step force checkpoints); else fmesh, mesh
  float* force_out[3] = {nullptr, nullptr, nullptr};
  fs2g_fft pm_fft_handle{};
  // binned deposit scratch (deposit_binned.cu)
  uint32_t* bin_counts = nullptr; uint32_t* bin_cursor = nullptr;
  int bin_tiles = 0;
  uint32_t* bin_idx = nullptr; size_t bin_cap = 0;
  uint32_t* bin_begin = nullptr; int* bin_overflow = nullptr;
  uint32_t* bin_tilewords = nullptr;   // len, olen, ostart, ocur: 4 per tile
  uint32_t* bin_ovf = nullptr;         // total, then 3 lists of bin_ovf_cap
  size_t bin_ovf_cap = 0;
  // what the counts in bin_counts were made for (the one-pass binning
  // reuses them): mesh, particles, shape; 0 particles = none
  int bin_prev_n = 0, bin_prev_shape = -1; size_t bin_prev_np = 0;
  bool bin_last_one_pass = false;      // the last deterministic deposit's binning
  int bin_shape_fixed = -1;            // -1: autotune
  int bin_shape = -1;                  // the last deterministic deposit's
  int bin_tuned_n = 0; size_t bin_tuned_np = 0;   // what it was tuned for
  void* bin_temp = nullptr; size_t bin_temp_bytes = 0;

  fs2g::FFTPlans fft;
  // fused Poisson pipeline (fft_pipeline.cu)
  int fft_engine = FS2G_FFT_AUTO;
  bool fused = false;                  // engine in use for the current mesh
  bool keep_delta_k = false;
  int fft_tile = 8;                    // kz columns per tile (4 or 8)
  float2* fz_a = nullptr; float2* fz_b = nullptr; float2* fz_c = nullptr;
  float2* fz_d = nullptr;
  float4* f4 = nullptr;        // fused path's force mesh, (fx, fy, fz, 0) per cell
  float2* fz_tw = nullptr;
  float2* fz_dk = nullptr;             // delta(k), pitch fused_pitch(n), if kept
  bool dk_valid = false;
  // the density mesh already holds the atomic deposit's starting value (-1
  // everywhere): the fused force reset it, and nothing has written it since
  bool mesh_prefilled = false;

  // timing
  bool timing = false;
  std::vector<fs2g::StageEvent> pending;
  std::vector<cudaEvent_t> event_pool;
  double stage_ms[fs2g::ST_NSTAGES] = {0};
  long stage_launches[fs2g::ST_NSTAGES] = {0};
};

struct fs2g_particles {
  fs2g_ctx* ctx = nullptr;
  size_t np_local = 0;
  size_t np_alloc = 0;
  size_t stride = 0;         // plane stride in floats (>= np_alloc, 32-aligned)
  uint64_t np_total = 0;
  double boxsize = 0.0;
  double a_x = 0.0, a_v = 0.0, a_f = 0.0;
  float* d_planes = nullptr; // 15 planes: x0..2 v0..2 dx1_0..2 dx2_0..2 f0..2
  uint64_t* d_id = nullptr;

  float* plane(int field, int c) const {
    return d_planes + (size_t)(3*field + c)*stride;
  }
};

struct fs2g_power {
  int n = 0;
  std::vector<double> log_k, log_P;
  // natural cubic spline of log P(log k): on [log_k[j], log_k[j+1])
  // log P = a + t(b + t(c + t d)), t = log k - log_k[j]
  std::vector<double> sa, sb, sc, sd;
  double eval_logP(double logk) const;
};

namespace fs2g {

// ---------------------------------------------------------------------
// context helpers (api.cu)
// ---------------------------------------------------------------------
void device_scope(fs2g_ctx* ctx);           // cudaSetDevice(ctx->device)
void check_device_error(fs2g_ctx* ctx);     // sync + read d_err, throws
void stage_begin(fs2g_ctx* ctx, int stage, cudaEvent_t* start);
void stage_end(fs2g_ctx* ctx, int stage, cudaEvent_t start);
struct StageScope {
  fs2g_ctx* ctx; int stage; cudaEvent_t start = nullptr;
  StageScope(fs2g_ctx* c, int s) : ctx(c), stage(s) { stage_begin(c, s, &start); }
  ~StageScope() { stage_end(ctx, stage, start); }
};
// particles per member of a batched context (np_local for batch 1)
inline size_t member_np(const fs2g_ctx* ctx, const fs2g_particles* p) {
  return p->np_local/(size_t) ctx->batch;
}
// every plan made for a context transforms ctx->batch stacked meshes
cufftHandle get_plan(fs2g_ctx* ctx, int kind, int n);
void fft_exec_r2c(fs2g_ctx* ctx, int n, float* in, float2* out);
void fft_exec_c2r_inplace(fs2g_ctx* ctx, int n, float2* data);
void* dmalloc(size_t bytes, const char* what);
void dfree(void* p);

// ---------------------------------------------------------------------
// cosmology (cosmology.cpp), host FP64
// ---------------------------------------------------------------------
void cosmology_init(double omega_m);
bool cosmology_initialised();
double cosmology_omega_m();
double cosmology_D_growth(double a);
double cosmology_D2_growth(double a, double D);
double cosmology_Dv_growth(double a, double D);
double cosmology_D2v_growth(double a, double D2);
double cosmology_D2a_growth(double D1, double D2);
double cosmology_f_growth_rate(double a);
double cosmology_hubble_function(double a);
double cosmology_omega(double a);
double cola_Sq(double ai, double af, double av);   // py/cola.cpp:157-179
double leapfrog_Sphi(double ai, double af);        // py/leapfrog.cpp:103-121
double leapfrog_Sq(double ai, double af);          // py/leapfrog.cpp:129-146

// ---------------------------------------------------------------------
// kernels (launchers)
// ---------------------------------------------------------------------
// pm_kernels.cu
void launch_wrap(fs2g_ctx* ctx, fs2g_particles* p);
// pm_kernels.cu: the atomic deposit onto a mesh that holds -1 (cleared by
// launch_clear_density, or reset by the fused force's XX pass).  wrap: fold
// the positions into the particles' box first, as launch_wrap does, in the
// same pass
void launch_clear_density(fs2g_ctx* ctx, float* mesh, int n);
void launch_deposit_atomic(fs2g_ctx* ctx, fs2g_particles* p, float* mesh,
                           int n, float boxsize, float fac, bool wrap = false);
// binned deposit (deposit_binned.cu): tiles of tx x ty x tz cells
// (clipped to n), one bin of particle indices per tile.  BIN_SHAPES tile
// shapes are built; shape 0 (BIN_TX x BIN_TY x BIN_TZ) is the default and
// the allocation-free entry point's.  Every shape gives the same bits.
constexpr int BIN_TX = 16, BIN_TY = 16, BIN_TZ = 32;
constexpr int BIN_SHAPES = 5;
struct BinGeom { int n, shape, tx, ty, tz, ntx, nty, ntz; };
BinGeom bin_geometry(int n, int shape = 0);
// scratch of the binned deposit: counts and cursor hold one word per tile,
// idx at least 8 np entries (the most bins np particles can touch)
struct BinScratch {
  uint32_t* counts; uint32_t* cursor; uint32_t* idx;
  void* temp; size_t temp_bytes;    // CUB scan storage, bin_scan_temp_bytes
  // the one-pass binning (reuse): bin starts, one word per tile, the
  // overflow flag, and the entries idx holds
  uint32_t* begin = nullptr; int* overflow = nullptr; size_t idx_cap = 0;
  // per tile: entries stored in the bin, overflow entries, their start and
  // a cursor; the overflow list (tile, particle) and its binned copy
  uint32_t* len = nullptr; uint32_t* olen = nullptr;
  uint32_t* ostart = nullptr; uint32_t* ocur = nullptr;
  uint32_t* ovf_total = nullptr; uint32_t* ovf_tile = nullptr;
  uint32_t* ovf_idx = nullptr; uint32_t* ovf_sorted = nullptr;
  size_t ovf_cap = 0;
};
size_t bin_scan_temp_bytes(int ntiles);
int fixed_point_shift(size_t np, float fac);
// clear-free deterministic deposit: every cell of the padded mesh's n^3
// region is written (-1 + sum) with the order-independent fixed-point
// accumulator (bitwise reproducible).  reuse: sc.counts holds the counts of
// a deposit of the same np particles with the same mesh, batch and shape
// (the previous one); the particles are binned in one pass into bins sized
// from them, with the two-pass binning as the fallback on the device.  wrap: fold positions into the box
// first (stored back).  err: device error word (a position below -1 cell
// is flagged there and skipped).
cudaError_t deposit_binned_on(cudaStream_t stream, float* x0, float* x1,
                              float* x2, size_t np, float* mesh, int n,
                              float dx_inv, float fac, float boxsize,
                              bool wrap, const BinScratch& sc, int* err,
                              int batch = 1, int shape = 0,
                              bool reuse = false);
// the shared-memory limits of every shape's deposit kernel
cudaError_t deposit_binned_set_smem_limits();
// fused Poisson pipeline (fft_pipeline.cu)
struct FusedBufs {
  const float* delta;  // density in
  float2 *A, *B, *C, *D;
  float4* f4;          // force mesh out: (f_x, f_y, f_z, 0) per cell, [n][n][n]
  float2* dk_out; const float2* tw; int n, pc; float f1;
  int tile;            // kz columns per tile of the y / x passes: 4 or 8
  // the density mesh (n x n x (n + 2) floats), reset to -1 by the XX pass
  // once FZ has read it, if fused_fills_mesh(); null: left as it is
  float* fill_mesh = nullptr;
};
bool fused_fills_mesh(const FusedBufs& f);
int fused_pitch(int n);
bool fused_supported(int n);
void fused_init_constants();
void fused_twiddles(int n, std::vector<float2>& out);
void launch_fused_pass(cudaStream_t s, int pass, const FusedBufs& f);
// one n = 1024 register-direct pass on a slab (fs2g_fused_pass_probe);
// average ms over `reps` launches
float fused_pass_probe(int pass, int planes, int reps);
// the three axes at once (k_force_k3): fk[a] = axis a's spectrum
void launch_force_k3(fs2g_ctx* ctx, const float2* delta_k, float2* const fk[3],
                     int n, float f1);
void launch_gather3(fs2g_ctx* ctx, fs2g_particles* p, const float* fx,
                    const float* fy, const float* fz, int n, float boxsize);
void launch_gather4(fs2g_ctx* ctx, fs2g_particles* p, const float4* f4, int n,
                    float boxsize);
void launch_extract_component(fs2g_ctx* ctx, const float4* f4, int comp,
                              float* dense, int n);
struct KickCoef;
struct DriftCoef;
void launch_fill_test_data(fs2g_ctx* ctx, float* fx, int n);
void launch_unpad(fs2g_ctx* ctx, const float* padded, float* dense, int n);
void launch_density_sum(fs2g_ctx* ctx, const float* mesh, int n,
                        double* d_sum);
// cola_kernels.cu
struct KickCoef { double neg15om; float kick_factor, q1, q2; };
struct DriftCoef { double dt; float da1, da2; };
// gather, then the step's kick and drift in the same pass (fs2g_cola_step)
void launch_gather4_kick_drift(fs2g_ctx* ctx, fs2g_particles* p,
                               const float4* f4, int n, float boxsize,
                               KickCoef k, DriftCoef d);
void launch_kick(fs2g_ctx* ctx, fs2g_particles* p, KickCoef k);
void launch_drift(fs2g_ctx* ctx, fs2g_particles* p, DriftCoef d);
void launch_kick_drift(fs2g_ctx* ctx, fs2g_particles* p, KickCoef k,
                       DriftCoef d);
// leapfrog (non-COLA) streams, py/leapfrog.cpp:18-95
void launch_leapfrog_velocity(fs2g_ctx* ctx, fs2g_particles* p, float dv,
                              float d2v);
void launch_leapfrog_kick(fs2g_ctx* ctx, fs2g_particles* p, double neg15om,
                          float kick_factor);
void launch_leapfrog_drift(fs2g_ctx* ctx, fs2g_particles* p, double dt);
// mode 0: dst plane c = v_c + c1 dx1_c + c2 dx2_c; mode 1: dst = c1 dx1_c
void launch_linear3(fs2g_ctx* ctx, fs2g_particles* p, float* dst,
                    size_t dst_stride, float c1, float c2, int mode);
// lpt_kernels.cu
struct SplineDev { const double* knots; const double* coef; int n; };
void launch_lpt_psi_k(fs2g_ctx* ctx, int nc, double boxsize,
                      unsigned long long seed, const double* u_phase,
                      const double* u_ampl, SplineDev ps, float2* psi0,
                      float2* psi1, float2* psi2);
void launch_lpt_psi_from_delta(fs2g_ctx* ctx, int nc, double boxsize,
                               const float2* delta_k, float2* psi0,
                               float2* psi1, float2* psi2);
void launch_lpt_psi_ij(fs2g_ctx* ctx, int nc, double boxsize,
                       float2* const psi[3], float2* const out[6]);
void launch_lpt_source(fs2g_ctx* ctx, int nc, float* const ij[6],
                       float* div);
void launch_lpt_psi2_k(fs2g_ctx* ctx, int nc, double boxsize,
                       const float2* div_k, float2* const out[3]);
void launch_lpt_particles(fs2g_ctx* ctx, fs2g_particles* p, int nc,
                          double boxsize, float offset,
                          float* const psi[3], float* const psi2[3],
                          float D1, float D2, float Dv, float D2v);
void lpt_draws_host(int nc, unsigned long long seed, double* u_phase,
                    double* u_ampl);

}  // namespace fs2g
