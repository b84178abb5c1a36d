// ensemble.cu -- many differentiable COLA runs of uneven sizes, replayed as
// one CUDA graph.
//
// Each member is one realisation: its own context (stream, PM buffers,
// cuFFT plans and work area) and its own differentiable run (api_diff.cu).
// A run of the ensemble is, per member: forward (2LPT from white noise,
// nsteps COLA steps, CIC density), the loss mean((delta - target)^2) and its
// gradient 2 (delta - target) / n^3, and the backward (the gradient with
// respect to the white noise).
//
// Graph mode forks every member's stream off the caller's stream, captures
// the members' work once and replays it with a single cudaGraphLaunch, so
// that the small members' kernels run side by side instead of one after
// another.  Loop mode runs the members one after another on the caller's
// stream: the plain path, looped.  Before the first run every member runs
// once eagerly, so that PM buffers, cuFFT plans and sort scratch exist
// before any capture.
//
// The autotuner times forward + backward of the first member of each size
// with each FFT engine and tile width that size allows (fused pipeline with
// 8 or 4 kz columns per tile, cuFFT) and gives every member of that size
// the fastest.
#include <algorithm>
#include <map>
#include <tuple>
#include <vector>
#include "internal.h"

using namespace fs2g;

struct fs2g_ensemble {
  struct Member {
    fs2g_ctx* ctx = nullptr;
    fs2g_diff* diff = nullptr;
    int nc = 0, n = 0;
    double L = 0;
    float* w = nullptr;          // white noise in, nc^3
    float* target = nullptr;     // target density, n^3
    float* delta = nullptr;      // density out, n^3
    float* dbar = nullptr;       // loss gradient wrt delta, n^3
    float* wbar = nullptr;       // gradient out, nc^3
    double* part = nullptr;      // the loss's block partials
    int engine = FS2G_FFT_AUTO, tile = 8;
    double tuned_ms = 0;
  };
  fs2g_ctx* main = nullptr;
  std::vector<Member> m;
  double* d_loss = nullptr;      // one per member
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join;
  cudaGraphExec_t exec = nullptr;
  long graph_kernels = 0;        // kernel nodes of the captured graph
  bool warmed = false;
};

namespace {

constexpr int TPB = 256;

constexpr int MSE_BLOCKS = 512;   // fixed: the loss's summation order

// dbar = 2 (delta - target) / cells; part[block] = that block's sum of
// (delta - target)^2 (a grid of MSE_BLOCKS blocks, fixed order)
__global__ void __launch_bounds__(TPB)
k_mse(const float* __restrict__ delta, const float* __restrict__ target,
      size_t cells, float* __restrict__ dbar, double* __restrict__ part) {
  __shared__ double warp_sum[TPB/32];
  double s = 0.0;
  const float inv = 1.0f/(float) cells;
  for(size_t i = blockIdx.x*(size_t) blockDim.x + threadIdx.x; i < cells;
      i += (size_t) gridDim.x*blockDim.x) {
    const float d = delta[i] - target[i];
    dbar[i] = 2.0f*d*inv;
    s += (double) d*(double) d;
  }
  for(int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if((threadIdx.x & 31) == 0) warp_sum[threadIdx.x >> 5] = s;
  __syncthreads();
  if(threadIdx.x == 0) {
    double t = 0.0;
    for(int w = 0; w < TPB/32; w++) t += warp_sum[w];
    part[blockIdx.x] = t;
  }
}

// loss = sum of the block partials in block order / cells (one thread)
__global__ void k_mse_total(const double* __restrict__ part, size_t cells,
                            double* __restrict__ loss) {
  double t = 0.0;
  for(int b = 0; b < MSE_BLOCKS; b++) t += part[b];
  *loss = t/(double) cells;
}

size_t cells3(int n) { return (size_t) n*n*n; }

// forward, loss, backward of member i on its context's current stream
void member_body(fs2g_ensemble* e, int i) {
  auto& mb = e->m[i];
  fs2g_ctx* c = mb.ctx;
  if(fs2g_diff_forward(mb.diff, mb.w, mb.delta) != FS2G_OK)
    throw Error{FS2G_ERR_RUNTIME, fs2g_last_error()};
  const size_t cells = cells3(mb.n);
  k_mse<<<MSE_BLOCKS, TPB, 0, c->stream>>>(mb.delta, mb.target, cells, mb.dbar,
                                           mb.part);
  FS2G_LAUNCHED(c);
  k_mse_total<<<1, 1, 0, c->stream>>>(mb.part, cells, e->d_loss + i);
  FS2G_LAUNCHED(c);
  if(fs2g_diff_backward(mb.diff, mb.dbar, mb.wbar) != FS2G_OK)
    throw Error{FS2G_ERR_RUNTIME, fs2g_last_error()};
}

void set_engine(fs2g_ensemble::Member& mb, int engine, int tile) {
  mb.engine = engine; mb.tile = tile;
  fs2g_pm_set_fft_engine(mb.ctx, engine);
  fs2g_pm_set_fft_tile(mb.ctx, tile);
  fs2g_pm_free(mb.ctx);                 // the next forward re-initialises
}

void drop_graph(fs2g_ensemble* e) {
  if(e->exec) { cudaGraphExecDestroy(e->exec); e->exec = nullptr; }
}

void autotune(fs2g_ensemble* e) {
  std::map<std::tuple<int, int, double>, std::vector<int>> groups;
  for(int i = 0; i < (int) e->m.size(); i++)
    groups[{e->m[i].nc, e->m[i].n, e->m[i].L}].push_back(i);
  for(auto& kv : groups) {
    auto& first = e->m[kv.second.front()];
    std::vector<std::pair<int, int>> cand;
    if(fused_supported(first.n)) cand = {{FS2G_FFT_FUSED, 8}, {FS2G_FFT_FUSED, 4}};
    cand.push_back({FS2G_FFT_CUFFT, 8});
    double best = 1e300;
    std::pair<int, int> pick = cand.front();
    cudaEvent_t t0, t1;
    FS2G_CUDA(cudaEventCreate(&t0));
    FS2G_CUDA(cudaEventCreate(&t1));
    for(auto& cd : cand) {
      set_engine(first, cd.first, cd.second);
      member_body(e, kv.second.front());        // initialise, warm
      float best_c = 1e30f;
      for(int r = 0; r < 3; r++) {
        FS2G_CUDA(cudaEventRecord(t0, first.ctx->stream));
        member_body(e, kv.second.front());
        FS2G_CUDA(cudaEventRecord(t1, first.ctx->stream));
        FS2G_CUDA(cudaEventSynchronize(t1));
        float ms = 0;
        FS2G_CUDA(cudaEventElapsedTime(&ms, t0, t1));
        best_c = std::min(best_c, ms);
      }
      if(best_c < best) { best = best_c; pick = cd; }
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    for(int i : kv.second) {
      set_engine(e->m[i], pick.first, pick.second);
      e->m[i].tuned_ms = best;
    }
  }
}

void release(fs2g_ensemble* e) {
  drop_graph(e);
  for(auto& mb : e->m) {
    if(mb.ctx) cudaStreamSynchronize(mb.ctx->stream);
    if(mb.diff) fs2g_diff_free(mb.diff);
    dfree(mb.w); dfree(mb.target); dfree(mb.delta); dfree(mb.dbar);
    dfree(mb.wbar); dfree(mb.part);
    if(mb.ctx) fs2g_ctx_destroy(mb.ctx);
  }
  e->m.clear();
  dfree(e->d_loss);
  if(e->fork) cudaEventDestroy(e->fork);
  for(auto ev : e->join) cudaEventDestroy(ev);
  e->join.clear();
}

}  // namespace

extern "C" {

int fs2g_ensemble_create(fs2g_ctx* c, int count, const int* nc, const int* n,
                         const double* boxsize, const fs2g_power* ps,
                         double a_init, int nsteps, const double* a_vel,
                         const double* a_pos, int tune,
                         fs2g_ensemble** out) {
  if(!c || !nc || !n || !boxsize || !ps || !out || count <= 0)
    return fail(FS2G_ERR_VALUE, "null argument or empty ensemble");
  fs2g_ensemble* e = new fs2g_ensemble();
  try {
    device_scope(c);
    e->main = c;
    e->d_loss = (double*) dmalloc((size_t) count*sizeof(double), "ensemble losses");
    FS2G_CUDA(cudaMemset(e->d_loss, 0, (size_t) count*sizeof(double)));
    FS2G_CUDA(cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming));
    e->m.resize(count);
    e->join.resize(count, nullptr);
    for(int i = 0; i < count; i++) {
      auto& mb = e->m[i];
      mb.nc = nc[i]; mb.n = n[i]; mb.L = boxsize[i];
      if(fs2g_ctx_create(c->device, &mb.ctx) != FS2G_OK)
        throw Error{FS2G_ERR_RUNTIME, fs2g_last_error()};
      mb.ctx->deposit_mode = c->deposit_mode;
      if(fs2g_diff_create(mb.ctx, mb.nc, mb.n, mb.L, ps, a_init, nsteps, a_vel,
                          a_pos, &mb.diff) != FS2G_OK)
        throw Error{FS2G_ERR_VALUE, fs2g_last_error()};
      const size_t wb = cells3(mb.nc)*sizeof(float), db = cells3(mb.n)*sizeof(float);
      mb.w = (float*) dmalloc(wb, "ensemble noise");
      mb.wbar = (float*) dmalloc(wb, "ensemble gradient");
      mb.target = (float*) dmalloc(db, "ensemble target");
      mb.delta = (float*) dmalloc(db, "ensemble density");
      mb.dbar = (float*) dmalloc(db, "ensemble loss gradient");
      mb.part = (double*) dmalloc(MSE_BLOCKS*sizeof(double), "ensemble loss partials");
      FS2G_CUDA(cudaMemset(mb.w, 0, wb));
      FS2G_CUDA(cudaMemset(mb.wbar, 0, wb));
      FS2G_CUDA(cudaMemset(mb.target, 0, db));
      FS2G_CUDA(cudaMemset(mb.delta, 0, db));
      FS2G_CUDA(cudaMemset(mb.dbar, 0, db));
      FS2G_CUDA(cudaEventCreateWithFlags(&e->join[i], cudaEventDisableTiming));
      mb.engine = mb.ctx->fft_engine; mb.tile = mb.ctx->fft_tile;
    }
    if(tune) autotune(e);
    FS2G_CUDA(cudaDeviceSynchronize());
  }
  catch(const Error& err) {
    release(e);
    delete e;
    return fail(err.code, err.msg);
  }
  *out = e;
  return FS2G_OK;
}

int fs2g_ensemble_free(fs2g_ensemble* e) {
  if(!e) return FS2G_OK;
  cudaSetDevice(e->main->device);
  release(e);
  delete e;
  return FS2G_OK;
}

int fs2g_ensemble_size(const fs2g_ensemble* e, int* count) {
  if(!e || !count) return fail(FS2G_ERR_VALUE, "null argument");
  *count = (int) e->m.size();
  return FS2G_OK;
}

int fs2g_ensemble_member(fs2g_ensemble* e, int i, float** white_noise,
                         float** target, float** density, float** gradient,
                         int* nc, int* n) {
  if(!e) return fail(FS2G_ERR_VALUE, "null argument");
  if(i < 0 || i >= (int) e->m.size()) return fail(FS2G_ERR_VALUE, "no such member");
  auto& mb = e->m[i];
  if(white_noise) *white_noise = mb.w;
  if(target) *target = mb.target;
  if(density) *density = mb.delta;
  if(gradient) *gradient = mb.wbar;
  if(nc) *nc = mb.nc;
  if(n) *n = mb.n;
  return FS2G_OK;
}

int fs2g_ensemble_tuning(const fs2g_ensemble* e, int i, int* engine, int* tile,
                         double* ms) {
  if(!e) return fail(FS2G_ERR_VALUE, "null argument");
  if(i < 0 || i >= (int) e->m.size()) return fail(FS2G_ERR_VALUE, "no such member");
  if(engine) *engine = e->m[i].engine;
  if(tile) *tile = e->m[i].tile;
  if(ms) *ms = e->m[i].tuned_ms;
  return FS2G_OK;
}

int fs2g_ensemble_forward_member(fs2g_ensemble* e, int i) {
  if(!e) return fail(FS2G_ERR_VALUE, "null argument");
  if(i < 0 || i >= (int) e->m.size()) return fail(FS2G_ERR_VALUE, "no such member");
  return guarded([&] {
    device_scope(e->main);
    auto& mb = e->m[i];
    if(fs2g_diff_forward(mb.diff, mb.w, mb.delta) != FS2G_OK)
      throw Error{FS2G_ERR_RUNTIME, fs2g_last_error()};
    FS2G_CUDA(cudaStreamSynchronize(mb.ctx->stream));
    check_device_error(mb.ctx);
  });
}

int fs2g_ensemble_run(fs2g_ensemble* e, int mode) {
  if(!e) return fail(FS2G_ERR_VALUE, "null argument");
  if(mode != FS2G_ENSEMBLE_LOOP && mode != FS2G_ENSEMBLE_GRAPH)
    return fail(FS2G_ERR_VALUE, "unknown ensemble mode");
  return guarded([&] {
    device_scope(e->main);
    cudaStream_t s0 = e->main->stream;
    if(!e->warmed) {
      // every member once, eagerly: buffers, plans and scratch exist before
      // any capture
      for(int i = 0; i < (int) e->m.size(); i++) member_body(e, i);
      FS2G_CUDA(cudaDeviceSynchronize());
      e->warmed = true;
    }
    if(mode == FS2G_ENSEMBLE_LOOP) {
      for(int i = 0; i < (int) e->m.size(); i++) {
        auto& mb = e->m[i];
        mb.ctx->stream = s0;
        try { member_body(e, i); }
        catch(...) { mb.ctx->stream = mb.ctx->own_stream; throw; }
        mb.ctx->stream = mb.ctx->own_stream;
      }
      return;
    }
    if(!e->exec) {
      cudaGraph_t g = nullptr;
      FS2G_CUDA(cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal));
      try {
        FS2G_CUDA(cudaEventRecord(e->fork, s0));
        for(int i = 0; i < (int) e->m.size(); i++) {
          auto& mb = e->m[i];
          FS2G_CUDA(cudaStreamWaitEvent(mb.ctx->stream, e->fork, 0));
          member_body(e, i);
          FS2G_CUDA(cudaEventRecord(e->join[i], mb.ctx->stream));
          FS2G_CUDA(cudaStreamWaitEvent(s0, e->join[i], 0));
        }
      }
      catch(...) {
        cudaStreamEndCapture(s0, &g);
        if(g) cudaGraphDestroy(g);
        throw;
      }
      FS2G_CUDA(cudaStreamEndCapture(s0, &g));
      size_t nodes = 0;
      FS2G_CUDA(cudaGraphGetNodes(g, nullptr, &nodes));
      std::vector<cudaGraphNode_t> list(nodes);
      if(nodes) FS2G_CUDA(cudaGraphGetNodes(g, list.data(), &nodes));
      e->graph_kernels = 0;
      for(auto nd : list) {
        cudaGraphNodeType t;
        if(cudaGraphNodeGetType(nd, &t) == cudaSuccess &&
           t == cudaGraphNodeTypeKernel)
          e->graph_kernels++;
      }
      const cudaError_t ie = cudaGraphInstantiate(&e->exec, g, 0);
      cudaGraphDestroy(g);
      if(ie != cudaSuccess) { e->exec = nullptr; throw_cuda(ie, "graph instantiate", __FILE__, __LINE__); }
    }
    FS2G_CUDA(cudaGraphLaunch(e->exec, s0));
  });
}

int fs2g_ensemble_graph_kernels(const fs2g_ensemble* e, long* count) {
  if(!e || !count) return fail(FS2G_ERR_VALUE, "null argument");
  *count = e->graph_kernels;
  return FS2G_OK;
}

int fs2g_ensemble_losses(fs2g_ensemble* e, double* host) {
  if(!e || !host) return fail(FS2G_ERR_VALUE, "null argument");
  return guarded([&] {
    device_scope(e->main);
    FS2G_CUDA(cudaStreamSynchronize(e->main->stream));
    for(auto& mb : e->m) {
      FS2G_CUDA(cudaStreamSynchronize(mb.ctx->stream));
      check_device_error(mb.ctx);
    }
    FS2G_CUDA(cudaMemcpy(host, e->d_loss, e->m.size()*sizeof(double),
                         cudaMemcpyDeviceToHost));
  });
}

}  // extern "C"
