// api_diff.cu -- the differentiable COLA simulation (no reference
// counterpart): white noise w -> delta(k) = T(k) FFT(w) -> 2LPT particles ->
// nsteps COLA steps -> CIC density, and its adjoint, which maps a cotangent
// of the final density to the gradient with respect to w.
//
// The forward keeps (x, v) before every step (per-step checkpoints, 24 bytes
// per particle per step).  The backward walks the steps in reverse: it
// restores the step's state, recomputes the step's density and force meshes,
// then applies the transposed kick/drift, CIC gather, Poisson solve and CIC
// deposit (adjoint_kernels.cu), and finally the transposed 2LPT maps.
//
// When the three force meshes of every step fit in a quarter of the free
// device memory (and the force takes the cuFFT path), the forward writes
// them straight into per-step checkpoints instead and the backward skips
// the recomputation (deposit, R2C, the k-space force, three C2R and the
// gather per step); only the positions are folded into the box again.
// Larger runs (a 1024^3 mesh needs 12.9 GB per step) recompute.
//
// On a batched context (ctx->batch = B members of one size, the ensemble's
// size classes) one run carries B realisations: white noise, density and
// gradient are [B][side^3], every mesh is B stacked meshes and every
// kernel and transform covers all members at once.
#include <cmath>
#include <vector>
#include "internal.h"

namespace fs2g {
void launch_scatter3(fs2g_ctx*, fs2g_particles*, const float*, size_t, int,
                     float, float*, float*, float*);
void launch_deriv_gather(fs2g_ctx*, fs2g_particles*, const float*, size_t,
                         const float*, const float*, const float*,
                         const float4*, const float*, float, int, float, float*,
                         size_t);
void launch_poisson_adj_k(fs2g_ctx*, const float2*, const float2*,
                          const float2*, float2*, int, float);
void launch_cola_adj(fs2g_ctx*, float*, float*, float*, float*, float*,
                     size_t, size_t, float, float, float, float, float, float);
void launch_white_to_delta(fs2g_ctx*, float2*, int, double, SplineDev);
void launch_lpt_adj_to_mesh(fs2g_ctx*, const float*, const float*,
                            const float*, size_t, int, float, float,
                            float* const[3], float* const[3]);
void launch_lpt_adj_s(fs2g_ctx*, float2* const[3], float2*, int, double);
void launch_lpt_adj_source(fs2g_ctx*, int, float* const[6], const float*);
void launch_lpt_adj_w(fs2g_ctx*, float2* const[9], float2*, int, double,
                      SplineDev);
void launch_pad(fs2g_ctx*, const float*, float*, int, float);
void launch_unpad(fs2g_ctx*, const float*, float*, int);
// api.cu
void pm_step_force(fs2g_ctx* c, fs2g_particles* p);
void pm_step_density(fs2g_ctx* c, fs2g_particles* p);
KickCoef cola_kick_coef(double a_v, double a_x, double a_vel);
DriftCoef cola_drift_coef(double a_x, double a_v, double a_pos);
void particles_alloc_internal(fs2g_ctx* c, size_t np, double boxsize,
                              fs2g_particles** out);
}  // namespace fs2g

using namespace fs2g;

struct fs2g_diff {
  fs2g_ctx* c = nullptr;
  int nc = 0, n = 0, nsteps = 0;
  double L = 0, a_init = 0;
  std::vector<double> avel, apos;
  double* d_knots = nullptr; double* d_coef = nullptr; SplineDev ps{};
  float D1 = 0, D2 = 0;
  fs2g_particles* p = nullptr;
  float* ckpt = nullptr;        // nsteps x 6 planes x stride (x, v)
  float2* dk = nullptr;         // delta(k) of the last forward
  float* adj = nullptr;         // 15 planes: xbar vbar dx1bar dx2bar fbar
  float* gbar[3] = {nullptr, nullptr, nullptr};
  float2* gk[3] = {nullptr, nullptr, nullptr};
  float* dbar = nullptr;
  float2* lb[13] = {nullptr};
  float* fck = nullptr;         // nsteps x 3 force meshes, when they fit
  bool fck_valid = false;       // the last forward filled fck
  bool have_forward = false;
};

namespace {

// one complex (or padded real) mesh per member of the context's batch
size_t mesh_bytes(const fs2g_ctx* c, int n) {
  return (size_t) n*n*(n/2 + 1)*sizeof(float2)*(size_t) c->batch;
}

void diff_release(fs2g_diff* d) {
  if(d->p) { dfree(d->p->d_planes); dfree(d->p->d_id); delete d->p; d->p = nullptr; }
  dfree(d->ckpt); dfree(d->dk); dfree(d->adj); dfree(d->dbar); dfree(d->fck);
  dfree(d->d_knots); dfree(d->d_coef);
  for(int i = 0; i < 3; i++) { dfree(d->gbar[i]); dfree(d->gk[i]); }
  for(int i = 0; i < 13; i++) dfree(d->lb[i]);
}

// the step's (a_x, a_v) before step i of the schedule
void step_scale_factors(const fs2g_diff* d, int i, double* ax, double* av) {
  *ax = i == 0 ? d->a_init : d->apos[i - 1];
  *av = i == 0 ? d->a_init : d->avel[i - 1];
}

// psi(k) from delta(k) and the 2LPT particles (as lpt_impl, kind 'cola')
void lpt_forward(fs2g_diff* d) {
  fs2g_ctx* c = d->c;
  const int nc = d->nc;
  float2* psi[3] = {d->lb[0], d->lb[1], d->lb[2]};
  float2* ij[6] = {d->lb[3], d->lb[4], d->lb[5], d->lb[6], d->lb[7], d->lb[8]};
  launch_lpt_psi_from_delta(c, nc, d->L, d->dk, psi[0], psi[1], psi[2]);
  launch_lpt_psi_ij(c, nc, d->L, psi, ij);
  for(int i = 0; i < 6; i++) fft_exec_c2r_inplace(c, nc, ij[i]);
  float* ijr[6];
  for(int i = 0; i < 6; i++) ijr[i] = reinterpret_cast<float*>(ij[i]);
  launch_lpt_source(c, nc, ijr, ijr[3]);
  fft_exec_r2c(c, nc, ijr[3], ij[3]);
  float2* psi2[3] = {ij[0], ij[1], ij[2]};
  launch_lpt_psi2_k(c, nc, d->L, ij[3], psi2);
  for(int i = 0; i < 3; i++) {
    fft_exec_c2r_inplace(c, nc, psi[i]);
    fft_exec_c2r_inplace(c, nc, psi2[i]);
  }
  float* pr[3] = {reinterpret_cast<float*>(psi[0]), reinterpret_cast<float*>(psi[1]),
                  reinterpret_cast<float*>(psi[2])};
  float* qr[3] = {reinterpret_cast<float*>(psi2[0]), reinterpret_cast<float*>(psi2[1]),
                  reinterpret_cast<float*>(psi2[2])};
  launch_lpt_particles(c, d->p, nc, d->L, 0.5f, pr, qr, d->D1, d->D2, 0.f, 0.f);
  d->p->np_local = (size_t) nc*nc*nc*(size_t) c->batch;
  d->p->np_total = d->p->np_local;
  d->p->a_x = d->p->a_v = d->a_init;
  d->p->a_f = 0.0;
}

}  // namespace

extern "C" {

int fs2g_diff_create(fs2g_ctx* c, int nc, int n, double boxsize,
                     const fs2g_power* ps, double a_init, int nsteps,
                     const double* a_vel, const double* a_pos,
                     fs2g_diff** out) {
  if(!c || !ps || !out || (nsteps > 0 && (!a_vel || !a_pos)))
    return fail(FS2G_ERR_VALUE, "null argument");
  if(nc < 4 || n < 4 || nsteps < 0 || !(boxsize > 0) || !(a_init > 0))
    return fail(FS2G_ERR_VALUE, "invalid differentiable-run parameters");
  fs2g_diff* d = new fs2g_diff();
  try {
    device_scope(c);
    if(!cosmology_initialised())
      throw Error{FS2G_ERR_RUNTIME, "cosmology module not initialised"};
    d->c = c; d->nc = nc; d->n = n; d->nsteps = nsteps; d->L = boxsize;
    d->a_init = a_init;
    d->avel.assign(a_vel, a_vel + nsteps);
    d->apos.assign(a_pos, a_pos + nsteps);
    const double dk = 2.0*M_PI/boxsize;
    const double kmax = std::sqrt(3.0)*dk*std::max(1, nc/2 - 1);
    if(std::log(dk) < ps->log_k.front() || std::log(kmax) > ps->log_k.back())
      throw Error{FS2G_ERR_VALUE, "power spectrum table does not cover the modes"};
    const int m = ps->n - 1;
    std::vector<double> cf(4*(size_t) m);
    for(int j = 0; j < m; j++) {
      cf[j] = ps->sa[j]; cf[m + j] = ps->sb[j];
      cf[2*m + j] = ps->sc[j]; cf[3*m + j] = ps->sd[j];
    }
    d->d_knots = (double*) dmalloc(ps->n*sizeof(double), "spline");
    d->d_coef = (double*) dmalloc(cf.size()*sizeof(double), "spline");
    FS2G_CUDA(cudaMemcpy(d->d_knots, ps->log_k.data(), ps->n*sizeof(double),
                         cudaMemcpyHostToDevice));
    FS2G_CUDA(cudaMemcpy(d->d_coef, cf.data(), cf.size()*sizeof(double),
                         cudaMemcpyHostToDevice));
    d->ps = SplineDev{d->d_knots, d->d_coef, ps->n};
    d->D1 = (float) cosmology_D_growth(a_init);                 // py/lpt.cpp:156
    d->D2 = (float) cosmology_D2_growth(a_init, d->D1);         // py/lpt.cpp:157
    const size_t np = (size_t) nc*nc*nc*(size_t) c->batch;
    particles_alloc_internal(c, np, boxsize, &d->p);
    const size_t stride = d->p->stride;
    d->ckpt = (float*) dmalloc((size_t) std::max(nsteps, 1)*6*stride*sizeof(float),
                               "checkpoints");
    d->adj = (float*) dmalloc(15*stride*sizeof(float), "adjoint planes");
    d->dk = (float2*) dmalloc(mesh_bytes(c, nc), "delta(k)");
    for(int i = 0; i < 13; i++) d->lb[i] = (float2*) dmalloc(mesh_bytes(c, nc), "LPT mesh");
    for(int i = 0; i < 3; i++) {
      d->gbar[i] = (float*) dmalloc(mesh_bytes(c, n), "adjoint mesh");
      d->gk[i] = (float2*) dmalloc(mesh_bytes(c, n), "adjoint spectrum");
    }
    d->dbar = (float*) dmalloc(mesh_bytes(c, n), "density adjoint");
    // the PM module: n cells over the box, pm_factor n/nc
    if(fs2g_pm_init(c, n, (double) n/nc, boxsize) != FS2G_OK)
      throw Error{FS2G_ERR_RUNTIME, fs2g_last_error()};
    // per-step force meshes, if they fit (cuFFT path only: the fused
    // pipeline writes its own interleaved mesh)
    if(!c->fused && nsteps > 0) {
      size_t free_b = 0, total_b = 0;
      FS2G_CUDA(cudaMemGetInfo(&free_b, &total_b));
      const size_t need = (size_t) nsteps*3*mesh_bytes(c, n);
      if(need <= free_b/4) d->fck = (float*) dmalloc(need, "force checkpoints");
    }
  }
  catch(const Error& e) { diff_release(d); delete d; return fail(e.code, e.msg); }
  catch(const std::bad_alloc&) { diff_release(d); delete d; return fail(FS2G_ERR_MEMORY, "out of host memory"); }
  *out = d;
  return FS2G_OK;
}

int fs2g_diff_free(fs2g_diff* d) {
  if(!d) return FS2G_OK;
  cudaSetDevice(d->c->device);
  cudaStreamSynchronize(d->c->stream);
  diff_release(d);
  delete d;
  return FS2G_OK;
}

int fs2g_diff_forward(fs2g_diff* d, const float* w, float* delta_out) {
  if(!d || !w || !delta_out) return fail(FS2G_ERR_VALUE, "null argument");
  fs2g_ctx* c = d->c;
  try {
    device_scope(c);
    if(c->pm_nc != d->n)
      if(fs2g_pm_init(c, d->n, (double) d->n/d->nc, d->L) != FS2G_OK)
        throw Error{FS2G_ERR_RUNTIME, fs2g_last_error()};
    const int nc = d->nc;
    // delta(k) = T(k) R2C(w)
    {
      StageScope s(c, ST_LPT_K);
      launch_pad(c, w, reinterpret_cast<float*>(d->dk), nc, 1.0f);
      fft_exec_r2c(c, nc, reinterpret_cast<float*>(d->dk), d->dk);
      launch_white_to_delta(c, d->dk, nc, d->L, d->ps);
    }
    {
      StageScope s(c, ST_LPT_PARTICLES);
      lpt_forward(d);
    }
    const size_t stride = d->p->stride;
    for(int i = 0; i < d->nsteps; i++) {
      FS2G_CUDA(cudaMemcpyAsync(d->ckpt + (size_t) i*6*stride, d->p->d_planes,
                                6*stride*sizeof(float), cudaMemcpyDeviceToDevice,
                                c->stream));
      if(d->fck && !c->fused) {
        float* f = d->fck + (size_t) i*3*(mesh_bytes(c, d->n)/sizeof(float));
        const size_t m = mesh_bytes(c, d->n)/sizeof(float);
        c->force_out[0] = f; c->force_out[1] = f + m; c->force_out[2] = f + 2*m;
      }
      try { pm_step_force(c, d->p); }
      catch(...) { c->force_out[0] = c->force_out[1] = c->force_out[2] = nullptr; throw; }
      c->force_out[0] = c->force_out[1] = c->force_out[2] = nullptr;
      const KickCoef k = cola_kick_coef(d->p->a_v, d->p->a_x, d->avel[i]);
      const DriftCoef dr = cola_drift_coef(d->p->a_x, d->avel[i], d->apos[i]);
      {
        StageScope s(c, ST_KICK_DRIFT);
        launch_kick_drift(c, d->p, k, dr);
      }
      d->p->a_v = d->avel[i];
      d->p->a_x = d->apos[i];
    }
    d->fck_valid = d->fck && !c->fused && d->nsteps > 0;
    pm_step_density(c, d->p);                       // wraps, then deposits
    launch_unpad(c, c->mesh, delta_out, d->n);
    d->have_forward = true;
    return FS2G_OK;
  }
  catch(const Error& e) { return fail(e.code, e.msg); }
}

int fs2g_diff_backward(fs2g_diff* d, const float* delta_bar, float* w_bar) {
  if(!d || !delta_bar || !w_bar) return fail(FS2G_ERR_VALUE, "null argument");
  if(!d->have_forward) return fail(FS2G_ERR_RUNTIME, "backward before forward");
  fs2g_ctx* c = d->c;
  try {
    device_scope(c);
    const int n = d->n, nc = d->nc;
    fs2g_particles* p = d->p;
    const size_t stride = p->stride, np = p->np_local;
    const float L = c->pm_boxsize;
    const float fac = (float)(c->pm_factor*c->pm_factor*c->pm_factor);
    const float f1 = (float)(-1.0/std::pow((double) n, 3.0)/(2.0*M_PI/(double) L));
    float* xb = d->adj;
    float* vb = d->adj + 3*stride;
    float* d1b = d->adj + 6*stride;
    float* d2b = d->adj + 9*stride;
    float* fb = d->adj + 12*stride;
    FS2G_CUDA(cudaMemsetAsync(d->adj, 0, 15*stride*sizeof(float), c->stream));
    // final density: particles hold the wrapped final positions
    launch_pad(c, delta_bar, d->dbar, n, 1.0f);
    launch_deriv_gather(c, p, nullptr, 0, nullptr, nullptr, nullptr, nullptr,
                        d->dbar, fac, n, L, xb, stride);
    for(int i = d->nsteps - 1; i >= 0; i--) {
      double ax, av;
      step_scale_factors(d, i, &ax, &av);
      FS2G_CUDA(cudaMemcpyAsync(p->d_planes, d->ckpt + (size_t) i*6*stride,
                                6*stride*sizeof(float), cudaMemcpyDeviceToDevice,
                                c->stream));
      p->a_x = ax; p->a_v = av; p->a_f = 0.0;
      const float* gm[3] = {c->fmesh[0], c->fmesh[1], c->mesh};
      if(d->fck_valid) {
        // the forward's force meshes of this step; x folded into the box
        // as the forward's deposit did
        launch_wrap(c, p);
        const size_t m = mesh_bytes(c, n)/sizeof(float);
        const float* f = d->fck + (size_t) i*3*m;
        gm[0] = f; gm[1] = f + m; gm[2] = f + 2*m;
      }
      else pm_step_force(c, p);     // x wrapped in place; force meshes kept
      const KickCoef k = cola_kick_coef(av, ax, d->avel[i]);
      const DriftCoef dr = cola_drift_coef(ax, d->avel[i], d->apos[i]);
      const float K = (float)(k.kick_factor*k.neg15om);
      launch_cola_adj(c, xb, vb, d1b, d2b, fb, stride, np, K, k.q1, k.q2,
                      (float) dr.dt, dr.da1, dr.da2);
      for(int a = 0; a < 3; a++)
        FS2G_CUDA(cudaMemsetAsync(d->gbar[a], 0, mesh_bytes(c, n), c->stream));
      launch_scatter3(c, p, fb, stride, n, L, d->gbar[0], d->gbar[1], d->gbar[2]);
      for(int a = 0; a < 3; a++) fft_exec_r2c(c, n, d->gbar[a], d->gk[a]);
      launch_poisson_adj_k(c, d->gk[0], d->gk[1], d->gk[2],
                           reinterpret_cast<float2*>(d->dbar), n, f1);
      fft_exec_c2r_inplace(c, n, reinterpret_cast<float2*>(d->dbar));
      launch_deriv_gather(c, p, fb, stride, gm[0], gm[1], gm[2],
                          c->fused && !d->fck_valid ? c->f4 : nullptr, d->dbar, fac,
                          n, L, xb, stride);
    }
    // 2LPT: psibar, psi2bar on the particle grid
    float* lr[13];
    for(int i = 0; i < 13; i++) lr[i] = reinterpret_cast<float*>(d->lb[i]);
    float* pm3[3] = {lr[0], lr[1], lr[2]};
    float* qm3[3] = {lr[3], lr[4], lr[5]};
    launch_lpt_adj_to_mesh(c, xb, d1b, d2b, stride, nc, d->D1, d->D2, pm3, qm3);
    for(int i = 3; i < 6; i++) fft_exec_r2c(c, nc, lr[i], d->lb[i]);
    float2* q3[3] = {d->lb[3], d->lb[4], d->lb[5]};
    launch_lpt_adj_s(c, q3, d->lb[6], nc, d->L);
    fft_exec_c2r_inplace(c, nc, d->lb[6]);                    // Sbar
    // recompute psi_ij(x) into lb3..5, lb10..12
    float2* psi[3] = {d->lb[7], d->lb[8], d->lb[9]};
    float2* ij[6] = {d->lb[3], d->lb[4], d->lb[5], d->lb[10], d->lb[11], d->lb[12]};
    launch_lpt_psi_from_delta(c, nc, d->L, d->dk, psi[0], psi[1], psi[2]);
    launch_lpt_psi_ij(c, nc, d->L, psi, ij);
    for(int i = 0; i < 6; i++) fft_exec_c2r_inplace(c, nc, ij[i]);
    float* ijr[6];
    for(int i = 0; i < 6; i++) ijr[i] = reinterpret_cast<float*>(ij[i]);
    launch_lpt_adj_source(c, nc, ijr, lr[6]);
    for(int i = 0; i < 3; i++) fft_exec_r2c(c, nc, lr[i], d->lb[i]);
    for(int i = 0; i < 6; i++) fft_exec_r2c(c, nc, ijr[i], ij[i]);
    float2* all[9] = {d->lb[0], d->lb[1], d->lb[2], ij[0], ij[1], ij[2], ij[3],
                      ij[4], ij[5]};
    launch_lpt_adj_w(c, all, d->lb[6], nc, d->L, d->ps);
    fft_exec_c2r_inplace(c, nc, d->lb[6]);
    launch_unpad(c, lr[6], w_bar, nc);
    // the particles now hold the first step's state: a second backward needs
    // a new forward
    d->have_forward = false;
    return FS2G_OK;
  }
  catch(const Error& e) { return fail(e.code, e.msg); }
}

int fs2g_diff_particles(fs2g_diff* d, fs2g_particles** p) {
  if(!d || !p) return fail(FS2G_ERR_VALUE, "null argument");
  *p = d->p;
  return FS2G_OK;
}

}  // extern "C"
