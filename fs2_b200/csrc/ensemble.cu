// ensemble.cu -- many differentiable COLA runs of uneven sizes, batched by
// size and replayed as one CUDA graph.
//
// A run of the ensemble is, per member (one realisation): forward (2LPT
// from white noise, nsteps COLA steps, CIC density), the loss
// mean((delta - target)^2) and its gradient 2 (delta - target) / n^3, and
// the backward (the gradient with respect to the white noise).
//
// Members of the same (nc, n, boxsize) form a size class.  A class runs as
// one or more chunks; a chunk is a batched context (ctx->batch members:
// stacked meshes, batched cuFFT plans, one particle set) with one batched
// differentiable run (api_diff.cu), so every kernel and transform of the
// chunk covers all of its members in a single launch.  The class's device
// buffers (noise, target, density, loss gradient, gradient) are [B][side^3]
// arrays; chunk k works on its slice of them.
//
// Graph mode forks every chunk onto its own stream off the caller's
// stream, captures the chunks' work once and replays it with a single
// cudaGraphLaunch, so the classes run side by side.  Loop mode is the plain
// path, looped: each member alone through its own unbatched context and
// differentiable run, one after another on the caller's stream (made on the
// first loop run).  Before the first graph capture every chunk runs once
// eagerly, so that buffers, plans and scratch exist.
//
// The autotuner picks, per class, the members per chunk -- B, B/2 or B/4
// (rounded up): fewer members per launch means more, smaller launches that
// run concurrently on separate streams -- by timing forward + loss +
// backward of the whole class with each and keeping the fastest.
#include <algorithm>
#include <map>
#include <tuple>
#include <vector>
#include "internal.h"

using namespace fs2g;

namespace {
struct Chunk {
  fs2g_ctx* ctx = nullptr;
  fs2g_diff* diff = nullptr;
  int first = 0, count = 0;      // the class's slots [first, first + count)
  cudaEvent_t join = nullptr;
};
struct Single {                  // one member alone (loop mode)
  fs2g_ctx* ctx = nullptr;
  fs2g_diff* diff = nullptr;
};
}  // namespace

struct fs2g_ensemble {
  struct Group {
    int nc = 0, n = 0;
    double L = 0;
    std::vector<int> members;    // member index of each slot
    float* w = nullptr;          // white noise, [B][nc^3]
    float* wbar = nullptr;       // gradient, [B][nc^3]
    float* target = nullptr;     // target density, [B][n^3]
    float* delta = nullptr;      // density, [B][n^3]
    float* dbar = nullptr;       // loss gradient wrt density, [B][n^3]
    double* part = nullptr;      // the loss's block partials, [B][MSE_BLOCKS]
    double* loss = nullptr;      // [B]
    std::vector<Chunk> chunks;
    int chunk_size = 0;
    double tuned_ms = 0;
  };
  fs2g_ctx* main = nullptr;
  fs2g_power ps;                 // a copy: loop-mode runs are made later
  double a_init = 0;
  int nsteps = 0;
  std::vector<double> avel, apos;
  int deposit_mode = FS2G_DEPOSIT_ATOMIC;
  std::vector<Group> g;
  std::vector<std::pair<int, int>> where;   // member -> (class, slot)
  std::vector<Single> single;
  cudaEvent_t fork = nullptr;
  cudaGraphExec_t exec = nullptr;
  long graph_kernels = 0;        // kernel nodes of the captured graph
  bool warmed = false;
};

namespace {

constexpr int TPB = 256;

constexpr int MSE_BLOCKS = 512;   // fixed: the loss's summation order

// member blockIdx.y of the launch: dbar = 2 (delta - target) / cells;
// part[block] = that block's sum of (delta - target)^2 (MSE_BLOCKS blocks
// per member, fixed order)
__global__ void __launch_bounds__(TPB)
k_mse(const float* __restrict__ delta, const float* __restrict__ target,
      size_t cells, float* __restrict__ dbar, double* __restrict__ part) {
  __shared__ double warp_sum[TPB/32];
  const size_t mo = blockIdx.y*cells;
  delta += mo; target += mo; dbar += mo;
  part += (size_t) blockIdx.y*MSE_BLOCKS;
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

// loss[b] = sum of member b's block partials in block order / cells (one
// thread per member)
__global__ void k_mse_total(const double* __restrict__ part, size_t cells,
                            int members, double* __restrict__ loss) {
  const int b = blockIdx.x*blockDim.x + threadIdx.x;
  if(b >= members) return;
  double t = 0.0;
  for(int k = 0; k < MSE_BLOCKS; k++) t += part[(size_t) b*MSE_BLOCKS + k];
  loss[b] = t/(double) cells;
}

size_t cells3(int n) { return (size_t) n*n*n; }

// loss and its gradient for `count` consecutive slots from `first`
void mse(fs2g_ensemble::Group& G, fs2g_ctx* c, int first, int count) {
  const size_t cells = cells3(G.n);
  const size_t o = (size_t) first*cells;
  k_mse<<<dim3(MSE_BLOCKS, count), TPB, 0, c->stream>>>(
      G.delta + o, G.target + o, cells, G.dbar + o,
      G.part + (size_t) first*MSE_BLOCKS);
  FS2G_LAUNCHED(c);
  k_mse_total<<<(count + 63)/64, 64, 0, c->stream>>>(
      G.part + (size_t) first*MSE_BLOCKS, cells, count, G.loss + first);
  FS2G_LAUNCHED(c);
}

void check(int rc) {
  if(rc != FS2G_OK) throw Error{FS2G_ERR_RUNTIME, fs2g_last_error()};
}

// forward, loss, backward of a chunk on its context's current stream
void chunk_body(fs2g_ensemble::Group& G, Chunk& ch) {
  const size_t cw = cells3(G.nc), cd = cells3(G.n);
  check(fs2g_diff_forward(ch.diff, G.w + ch.first*cw, G.delta + ch.first*cd));
  mse(G, ch.ctx, ch.first, ch.count);
  check(fs2g_diff_backward(ch.diff, G.dbar + ch.first*cd,
                           G.wbar + ch.first*cw));
}

// a context of `batch` members with its differentiable run
void make_run(fs2g_ensemble* e, int nc, int n, double L, int batch,
              fs2g_ctx** ctx, fs2g_diff** diff) {
  check(fs2g_ctx_create(e->main->device, ctx));
  (*ctx)->batch = batch;
  (*ctx)->deposit_mode = e->deposit_mode;
  if(fs2g_diff_create(*ctx, nc, n, L, &e->ps, e->a_init, e->nsteps,
                      e->avel.data(), e->apos.data(), diff) != FS2G_OK) {
    const Error err{FS2G_ERR_VALUE, fs2g_last_error()};
    fs2g_ctx_destroy(*ctx);
    *ctx = nullptr;
    throw err;
  }
}

void free_chunks(std::vector<Chunk>& chunks) {
  for(auto& ch : chunks) {
    if(ch.ctx) cudaStreamSynchronize(ch.ctx->stream);
    if(ch.diff) fs2g_diff_free(ch.diff);
    if(ch.ctx) fs2g_ctx_destroy(ch.ctx);
    if(ch.join) cudaEventDestroy(ch.join);
  }
  chunks.clear();
}

// the class's chunks of `size` members each (the last one may be smaller)
void make_chunks(fs2g_ensemble* e, fs2g_ensemble::Group& G, int size) {
  free_chunks(G.chunks);
  const int B = (int) G.members.size();
  try {
    for(int first = 0; first < B; first += size) {
      Chunk ch;
      ch.first = first;
      ch.count = std::min(size, B - first);
      FS2G_CUDA(cudaEventCreateWithFlags(&ch.join, cudaEventDisableTiming));
      G.chunks.push_back(ch);
      make_run(e, G.nc, G.n, G.L, ch.count, &G.chunks.back().ctx,
               &G.chunks.back().diff);
    }
  }
  catch(...) { free_chunks(G.chunks); throw; }
  G.chunk_size = size;
}

// every chunk of the class once, each on its own stream, joined back onto
// stream s0 (eager; the same fork/join the graph capture records)
void run_group(fs2g_ensemble* e, fs2g_ensemble::Group& G, cudaStream_t s0) {
  FS2G_CUDA(cudaEventRecord(e->fork, s0));
  for(auto& ch : G.chunks) {
    FS2G_CUDA(cudaStreamWaitEvent(ch.ctx->stream, e->fork, 0));
    chunk_body(G, ch);
    FS2G_CUDA(cudaEventRecord(ch.join, ch.ctx->stream));
    FS2G_CUDA(cudaStreamWaitEvent(s0, ch.join, 0));
  }
}

void drop_graph(fs2g_ensemble* e) {
  if(e->exec) { cudaGraphExecDestroy(e->exec); e->exec = nullptr; }
}

void autotune(fs2g_ensemble* e) {
  cudaStream_t s0 = e->main->stream;
  cudaEvent_t t0, t1;
  FS2G_CUDA(cudaEventCreate(&t0));
  FS2G_CUDA(cudaEventCreate(&t1));
  try {
    for(auto& G : e->g) {
      const int B = (int) G.members.size();
      std::vector<int> cand;
      for(int div : {1, 2, 4}) {
        const int sz = (B + div - 1)/div;
        if(std::find(cand.begin(), cand.end(), sz) == cand.end()) cand.push_back(sz);
      }
      double best = 1e300;
      int pick = cand.front();
      for(int sz : cand) {
        make_chunks(e, G, sz);
        run_group(e, G, s0);                  // initialise, warm
        float best_c = 1e30f;
        for(int r = 0; r < 2; r++) {
          FS2G_CUDA(cudaEventRecord(t0, s0));
          run_group(e, G, s0);
          FS2G_CUDA(cudaEventRecord(t1, s0));
          FS2G_CUDA(cudaEventSynchronize(t1));
          float ms = 0;
          FS2G_CUDA(cudaEventElapsedTime(&ms, t0, t1));
          best_c = std::min(best_c, ms);
        }
        if(best_c < best) { best = best_c; pick = sz; }
      }
      if(G.chunk_size != pick) make_chunks(e, G, pick);
      G.tuned_ms = best;
    }
  }
  catch(...) { cudaEventDestroy(t0); cudaEventDestroy(t1); throw; }
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
}

void release(fs2g_ensemble* e) {
  drop_graph(e);
  for(auto& G : e->g) {
    free_chunks(G.chunks);
    dfree(G.w); dfree(G.wbar); dfree(G.target); dfree(G.delta);
    dfree(G.dbar); dfree(G.part); dfree(G.loss);
  }
  e->g.clear();
  for(auto& s : e->single) {
    if(s.ctx) cudaStreamSynchronize(s.ctx->stream);
    if(s.diff) fs2g_diff_free(s.diff);
    if(s.ctx) fs2g_ctx_destroy(s.ctx);
  }
  e->single.clear();
  if(e->fork) { cudaEventDestroy(e->fork); e->fork = nullptr; }
}

// member i's slices of its class's buffers
struct View { fs2g_ensemble::Group* G; int slot; };
View view(fs2g_ensemble* e, int i) {
  return View{&e->g[e->where[i].first], e->where[i].second};
}

}  // namespace

extern "C" {

int fs2g_ensemble_create(fs2g_ctx* c, int count, const int* nc, const int* n,
                         const double* boxsize, const fs2g_power* ps,
                         double a_init, int nsteps, const double* a_vel,
                         const double* a_pos, int tune,
                         fs2g_ensemble** out) {
  if(!c || !nc || !n || !boxsize || !ps || !out || count <= 0 ||
     (nsteps > 0 && (!a_vel || !a_pos)))
    return fail(FS2G_ERR_VALUE, "null argument or empty ensemble");
  fs2g_ensemble* e = new fs2g_ensemble();
  try {
    device_scope(c);
    e->main = c;
    e->ps = *ps;
    e->a_init = a_init;
    e->nsteps = nsteps;
    e->avel.assign(a_vel, a_vel + std::max(nsteps, 0));
    e->apos.assign(a_pos, a_pos + std::max(nsteps, 0));
    e->deposit_mode = c->deposit_mode;
    FS2G_CUDA(cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming));
    // size classes in order of first appearance
    std::map<std::tuple<int, int, double>, int> cls;
    e->where.resize(count);
    for(int i = 0; i < count; i++) {
      const auto key = std::make_tuple(nc[i], n[i], boxsize[i]);
      auto it = cls.find(key);
      if(it == cls.end()) {
        it = cls.emplace(key, (int) e->g.size()).first;
        e->g.emplace_back();
        e->g.back().nc = nc[i]; e->g.back().n = n[i]; e->g.back().L = boxsize[i];
      }
      auto& G = e->g[it->second];
      e->where[i] = {it->second, (int) G.members.size()};
      G.members.push_back(i);
    }
    for(auto& G : e->g) {
      const size_t B = G.members.size();
      const size_t wb = B*cells3(G.nc)*sizeof(float), db = B*cells3(G.n)*sizeof(float);
      G.w = (float*) dmalloc(wb, "ensemble noise");
      G.wbar = (float*) dmalloc(wb, "ensemble gradient");
      G.target = (float*) dmalloc(db, "ensemble target");
      G.delta = (float*) dmalloc(db, "ensemble density");
      G.dbar = (float*) dmalloc(db, "ensemble loss gradient");
      G.part = (double*) dmalloc(B*MSE_BLOCKS*sizeof(double), "ensemble loss partials");
      G.loss = (double*) dmalloc(B*sizeof(double), "ensemble losses");
      FS2G_CUDA(cudaMemset(G.w, 0, wb));
      FS2G_CUDA(cudaMemset(G.wbar, 0, wb));
      FS2G_CUDA(cudaMemset(G.target, 0, db));
      FS2G_CUDA(cudaMemset(G.delta, 0, db));
      FS2G_CUDA(cudaMemset(G.dbar, 0, db));
      FS2G_CUDA(cudaMemset(G.loss, 0, B*sizeof(double)));
      make_chunks(e, G, (int) B);
    }
    if(tune) autotune(e);
    FS2G_CUDA(cudaDeviceSynchronize());
  }
  catch(const Error& err) {
    release(e);
    delete e;
    return fail(err.code, err.msg);
  }
  catch(const std::bad_alloc&) {
    release(e);
    delete e;
    return fail(FS2G_ERR_MEMORY, "out of host memory");
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
  *count = (int) e->where.size();
  return FS2G_OK;
}

int fs2g_ensemble_member(fs2g_ensemble* e, int i, float** white_noise,
                         float** target, float** density, float** gradient,
                         int* nc, int* n) {
  if(!e) return fail(FS2G_ERR_VALUE, "null argument");
  if(i < 0 || i >= (int) e->where.size()) return fail(FS2G_ERR_VALUE, "no such member");
  const View v = view(e, i);
  const size_t cw = cells3(v.G->nc)*v.slot, cd = cells3(v.G->n)*v.slot;
  if(white_noise) *white_noise = v.G->w + cw;
  if(target) *target = v.G->target + cd;
  if(density) *density = v.G->delta + cd;
  if(gradient) *gradient = v.G->wbar + cw;
  if(nc) *nc = v.G->nc;
  if(n) *n = v.G->n;
  return FS2G_OK;
}

int fs2g_ensemble_tuning(const fs2g_ensemble* e, int i, int* engine,
                         int* chunk, double* ms) {
  if(!e) return fail(FS2G_ERR_VALUE, "null argument");
  if(i < 0 || i >= (int) e->where.size()) return fail(FS2G_ERR_VALUE, "no such member");
  const auto& G = e->g[e->where[i].first];
  if(engine) *engine = G.chunks.empty() ? FS2G_FFT_CUFFT
                                        : (G.chunks.front().ctx->fused
                                           ? FS2G_FFT_FUSED : FS2G_FFT_CUFFT);
  if(chunk) *chunk = G.chunk_size;
  if(ms) *ms = G.tuned_ms;
  return FS2G_OK;
}

int fs2g_ensemble_forward_member(fs2g_ensemble* e, int i) {
  if(!e) return fail(FS2G_ERR_VALUE, "null argument");
  if(i < 0 || i >= (int) e->where.size()) return fail(FS2G_ERR_VALUE, "no such member");
  return guarded([&] {
    device_scope(e->main);
    const View v = view(e, i);
    auto& G = *v.G;
    // the forward of member i's chunk (every member of the chunk gets its
    // density; the others' results are of no concern here)
    for(auto& ch : G.chunks) {
      if(v.slot < ch.first || v.slot >= ch.first + ch.count) continue;
      check(fs2g_diff_forward(ch.diff, G.w + ch.first*cells3(G.nc),
                              G.delta + ch.first*cells3(G.n)));
      FS2G_CUDA(cudaStreamSynchronize(ch.ctx->stream));
      check_device_error(ch.ctx);
    }
  });
}

int fs2g_ensemble_run(fs2g_ensemble* e, int mode) {
  if(!e) return fail(FS2G_ERR_VALUE, "null argument");
  if(mode != FS2G_ENSEMBLE_LOOP && mode != FS2G_ENSEMBLE_GRAPH)
    return fail(FS2G_ERR_VALUE, "unknown ensemble mode");
  return guarded([&] {
    device_scope(e->main);
    cudaStream_t s0 = e->main->stream;
    if(mode == FS2G_ENSEMBLE_LOOP) {
      // the plain path: each member alone, one after another on s0
      if(e->single.empty()) {
        e->single.resize(e->where.size());
        for(size_t i = 0; i < e->where.size(); i++) {
          const auto& G = e->g[e->where[i].first];
          make_run(e, G.nc, G.n, G.L, 1, &e->single[i].ctx, &e->single[i].diff);
        }
      }
      for(size_t i = 0; i < e->where.size(); i++) {
        Single& s = e->single[i];
        const View v = view(e, (int) i);
        auto& G = *v.G;
        s.ctx->stream = s0;
        try {
          check(fs2g_diff_forward(s.diff, G.w + v.slot*cells3(G.nc),
                                  G.delta + v.slot*cells3(G.n)));
          mse(G, s.ctx, v.slot, 1);
          check(fs2g_diff_backward(s.diff, G.dbar + v.slot*cells3(G.n),
                                   G.wbar + v.slot*cells3(G.nc)));
        }
        catch(...) { s.ctx->stream = s.ctx->own_stream; throw; }
        s.ctx->stream = s.ctx->own_stream;
      }
      return;
    }
    if(!e->warmed) {
      // every chunk once, eagerly: buffers, plans and scratch exist before
      // the capture
      for(auto& G : e->g) run_group(e, G, s0);
      FS2G_CUDA(cudaStreamSynchronize(s0));
      e->warmed = true;
    }
    if(!e->exec) {
      cudaGraph_t g = nullptr;
      FS2G_CUDA(cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal));
      try {
        for(auto& G : e->g) {
          FS2G_CUDA(cudaEventRecord(e->fork, s0));
          for(auto& ch : G.chunks) {
            FS2G_CUDA(cudaStreamWaitEvent(ch.ctx->stream, e->fork, 0));
            chunk_body(G, ch);
            FS2G_CUDA(cudaEventRecord(ch.join, ch.ctx->stream));
          }
        }
        for(auto& G : e->g)
          for(auto& ch : G.chunks) FS2G_CUDA(cudaStreamWaitEvent(s0, ch.join, 0));
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
    for(auto& G : e->g)
      for(auto& ch : G.chunks) {
        FS2G_CUDA(cudaStreamSynchronize(ch.ctx->stream));
        check_device_error(ch.ctx);
      }
    for(auto& s : e->single) check_device_error(s.ctx);
    for(auto& G : e->g) {
      std::vector<double> l(G.members.size());
      FS2G_CUDA(cudaMemcpy(l.data(), G.loss, l.size()*sizeof(double),
                           cudaMemcpyDeviceToHost));
      for(size_t k = 0; k < l.size(); k++) host[G.members[k]] = l[k];
    }
  });
}

}  // extern "C"
