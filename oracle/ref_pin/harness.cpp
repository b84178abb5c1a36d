// harness.cpp -- C entry points into the reference's own PM / COLA / 2LPT
// code, compiled from its sources (py/pm.cpp, py/cola.cpp, py/lpt.cpp,
// py/fft.cpp, py/cosmology.cpp, py/power.cpp, ...) with the single-rank
// stand-ins of oracle/ref_pin/include and stubs.cpp.
//
// TEST INFRASTRUCTURE ONLY: loaded by tests/ (through oracle/ref.py) to pin
// the oracle's restatement to the reference's arithmetic; never part of the
// product.  Each entry point follows the reference's Python wrapper for the
// same call (py/py_pm.cpp, py/py_cola.cpp, py/py_lpt.cpp) on one rank.
//
// Arrays are [np][3] float rows, meshes [n][n][2(n/2+1)] floats, spectra
// [n][n][n/2+1] (re, im) float pairs in kx-major order (the reference's PM
// spectrum is stored ky-major, FFTW_MPI_TRANSPOSED_OUT; the harness
// converts).
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "comm.h"
#include "cola.h"
#include "config.h"
#include "cosmology.h"
#include "fft.h"
#include "lpt.h"
#include "mem.h"
#include "msg.h"
#include "particle.h"
#include "pm.h"
#include "power.h"
#include "util.h"

// ------------------------------------------------------------------
// py/pm_domain.cpp on one rank: the decomposition has no other domain
// (allocate_decomposition, :249-296, pushes n - 1 = 0 entries), so no
// particle is ever sent and the buffers the PM loops read are empty.
// Its one-sided MPI exchange is therefore not compiled; these are the
// accessors pm.cpp calls (:126-135, :330-335, :349-351).
// ------------------------------------------------------------------
Pos const* pm_domain_buffer_positions() { return nullptr; }
Float3* pm_domain_buffer_forces() { return nullptr; }
int pm_domain_buffer_np() { return 0; }

extern "C" {
typedef int (*fs2ref_fft_hook)(void* ctx, int inverse, int n0, int n1, int n2,
                               int transposed, float* real, float* cplx);
void fs2ref_set_fft_hooks(fs2ref_fft_hook before, fs2ref_fft_hook after,
                          void* ctx);
}

namespace {

double g_boxsize = 0.0;
int g_n = 0;

// FFT capture / injection around pm_compute_force's four transforms
struct ForceHooks {
  const float* dk_inject = nullptr;   // replaces the R2C output
  float* fk_capture = nullptr;        // 3 spectra: the C2R inputs
  float* mesh_capture = nullptr;      // 3 meshes: the C2R outputs
  const float* mesh_inject = nullptr; // 3 meshes: replace the C2R outputs
  int c2r_calls = 0;
};

size_t nk_of(int n) { return (size_t) n/2 + 1; }
size_t ncz_of(int n) { return 2*nk_of(n); }

// the PM spectrum is [ky][kx][kz] (transposed); convert to/from [kx][ky][kz]
void spectrum_to_kx_major(const float* t, float* out, int n, int transposed) {
  const size_t nk = nk_of(n);
  for(size_t kx = 0; kx < (size_t) n; kx++)
    for(size_t ky = 0; ky < (size_t) n; ky++)
      for(size_t kz = 0; kz < nk; kz++) {
        const size_t src = transposed ? (ky*n + kx)*nk + kz : (kx*n + ky)*nk + kz;
        const size_t dst = (kx*n + ky)*nk + kz;
        out[2*dst] = t[2*src];
        out[2*dst + 1] = t[2*src + 1];
      }
}

void spectrum_from_kx_major(const float* in, float* t, int n, int transposed) {
  const size_t nk = nk_of(n);
  for(size_t kx = 0; kx < (size_t) n; kx++)
    for(size_t ky = 0; ky < (size_t) n; ky++)
      for(size_t kz = 0; kz < nk; kz++) {
        const size_t dst = transposed ? (ky*n + kx)*nk + kz : (kx*n + ky)*nk + kz;
        const size_t src = (kx*n + ky)*nk + kz;
        t[2*dst] = in[2*src];
        t[2*dst + 1] = in[2*src + 1];
      }
}

int hook_before(void* ctx, int inverse, int n0, int, int, int transposed,
                float*, float* cplx) {
  ForceHooks* h = static_cast<ForceHooks*>(ctx);
  if(inverse && h->fk_capture) {
    const size_t K = (size_t) n0*n0*nk_of(n0);
    spectrum_to_kx_major(cplx, h->fk_capture + 2*K*h->c2r_calls, n0,
                         transposed);
  }
  return 0;
}

int hook_after(void* ctx, int inverse, int n0, int, int, int transposed,
               float* real, float* cplx) {
  ForceHooks* h = static_cast<ForceHooks*>(ctx);
  const size_t R = (size_t) n0*n0*ncz_of(n0);
  if(!inverse) {
    if(h->dk_inject) spectrum_from_kx_major(h->dk_inject, cplx, n0, transposed);
    return 0;
  }
  if(h->mesh_inject)
    std::memcpy(real, h->mesh_inject + R*h->c2r_calls, R*sizeof(float));
  if(h->mesh_capture)
    std::memcpy(h->mesh_capture + R*h->c2r_calls, real, R*sizeof(float));
  h->c2r_calls++;
  return 0;
}

Particles* make_particles(size_t np, double boxsize) {
  Particles* p = new Particles(np > 0 ? np : 1, boxsize);
  p->np_local = np;
  return p;
}

template<class F> int guarded(F f) {
  try { f(); return 0; }
  catch(...) { return -1; }
}

}  // namespace

extern "C" {

int fs2ref_version(void) { return 1; }

// comm_mpi_init (single rank), quiet messages, cosmology_init
// (py/py_package.cpp:160-180, py/py_cosmology.cpp)
int fs2ref_init(double omega_m) {
  return guarded([&] {
    comm_mpi_init(nullptr, nullptr);
    msg_set_loglevel(msg_fatal);
    cosmology_init(omega_m);
  });
}

double fs2ref_D_growth(double a) { return cosmology_D_growth(a); }
double fs2ref_D2_growth(double a, double D) { return cosmology_D2_growth(a, D); }
double fs2ref_Dv_growth(double a, double D) { return cosmology_Dv_growth(a, D); }
double fs2ref_D2v_growth(double a, double D2) { return cosmology_D2v_growth(a, D2); }

// py_pm_init, py/py_pm.cpp:10-31
int fs2ref_pm_init(int nc_pm, double pm_factor, double boxsize) {
  return guarded([&] {
    const size_t mem_size = fft_mem_size(nc_pm, 1);
    Mem* const mem1 = new Mem("ParticleMesh", mem_size);
    Mem* const mem2 = new Mem("delta_k", mem_size);
    pm_init(nc_pm, pm_factor, mem1, mem2, boxsize);
    g_boxsize = boxsize;
    g_n = nc_pm;
  });
}

// pm_domain_send_positions' wrap (one rank: only periodic_wrapup_p,
// py/pm_domain.cpp:113-114) when `wrap`, then pm_compute_density
// (py/pm.cpp:341-355).  x is updated in place; the density mesh (padded)
// is copied to mesh_out.
int fs2ref_pm_density(float* x, size_t np, int wrap, float* mesh_out) {
  return guarded([&] {
    Particles* p = make_particles(np, g_boxsize);
    for(size_t i = 0; i < np; i++)
      for(int k = 0; k < 3; k++) p->p[i].x[k] = x[3*i + k];
    if(wrap) util_periodic_wrapup(p);
    FFT* fft = pm_compute_density(p);
    std::memcpy(mesh_out, fft->fx, (size_t) g_n*g_n*ncz_of(g_n)*sizeof(float));
    for(size_t i = 0; i < np; i++)
      for(int k = 0; k < 3; k++) x[3*i + k] = p->p[i].x[k];
    delete p->pv; free(p->force); delete p;
  });
}

// fs2ref_pm_density followed by pm_compute_force (py/pm.cpp:306-338): f is
// [np][3].  Optional hooks: dk_inject replaces delta(k) after the R2C;
// fk_capture receives the three k-space force spectra that enter the C2R;
// mesh_capture the three force meshes that leave it; mesh_inject replaces
// those meshes before the gather reads them.
int fs2ref_pm_force(float* x, size_t np, int wrap, float* f,
                    const float* dk_inject, float* fk_capture,
                    float* mesh_capture, const float* mesh_inject) {
  return guarded([&] {
    Particles* p = make_particles(np, g_boxsize);
    for(size_t i = 0; i < np; i++)
      for(int k = 0; k < 3; k++) p->p[i].x[k] = x[3*i + k];
    if(wrap) util_periodic_wrapup(p);
    p->a_x = 1.0; p->a_f = 0.0;
    ForceHooks h;
    h.dk_inject = dk_inject; h.fk_capture = fk_capture;
    h.mesh_capture = mesh_capture; h.mesh_inject = mesh_inject;
    fs2ref_set_fft_hooks(hook_before, hook_after, &h);
    try {
      pm_compute_density(p);
      pm_compute_force(p);
    }
    catch(...) { fs2ref_set_fft_hooks(nullptr, nullptr, nullptr); throw; }
    fs2ref_set_fft_hooks(nullptr, nullptr, nullptr);
    for(size_t i = 0; i < np; i++)
      for(int k = 0; k < 3; k++) {
        f[3*i + k] = p->force[i][k];
        x[3*i + k] = p->p[i].x[k];
      }
    delete p->pv; free(p->force); delete p;
  });
}

// cola_kick (py/cola.cpp:48-92) on particles at (a_x, a_v): v updated
int fs2ref_cola_kick(float* v, const float* f, const float* dx1,
                     const float* dx2, size_t np, double a_x, double a_v,
                     double a_vel) {
  return guarded([&] {
    Particles* p = make_particles(np, 1.0);
    for(size_t i = 0; i < np; i++)
      for(int k = 0; k < 3; k++) {
        p->p[i].v[k] = v[3*i + k];
        p->p[i].dx1[k] = dx1[3*i + k];
        p->p[i].dx2[k] = dx2[3*i + k];
        p->force[i][k] = f[3*i + k];
      }
    p->a_x = a_x; p->a_v = a_v;
    cola_kick(p, a_vel);
    for(size_t i = 0; i < np; i++)
      for(int k = 0; k < 3; k++) v[3*i + k] = p->p[i].v[k];
    delete p->pv; free(p->force); delete p;
  });
}

// cola_drift (py/cola.cpp:94-127): x updated
int fs2ref_cola_drift(float* x, const float* v, const float* dx1,
                      const float* dx2, size_t np, double a_x, double a_v,
                      double a_pos) {
  return guarded([&] {
    Particles* p = make_particles(np, 1.0);
    for(size_t i = 0; i < np; i++)
      for(int k = 0; k < 3; k++) {
        p->p[i].x[k] = x[3*i + k];
        p->p[i].v[k] = v[3*i + k];
        p->p[i].dx1[k] = dx1[3*i + k];
        p->p[i].dx2[k] = dx2[3*i + k];
      }
    p->a_x = a_x; p->a_v = a_v;
    cola_drift(p, a_pos);
    for(size_t i = 0; i < np; i++)
      for(int k = 0; k < 3; k++) x[3*i + k] = p->p[i].x[k];
    delete p->pv; free(p->force); delete p;
  });
}

// cola_velocity (py/cola.cpp:129-148) at a_x
int fs2ref_cola_velocity(const float* v, const float* dx1, const float* dx2,
                         size_t np, double a_x, float* out) {
  return guarded([&] {
    Particles* p = make_particles(np, 1.0);
    for(size_t i = 0; i < np; i++)
      for(int k = 0; k < 3; k++) {
        p->p[i].v[k] = v[3*i + k];
        p->p[i].dx1[k] = dx1[3*i + k];
        p->p[i].dx2[k] = dx2[3*i + k];
      }
    p->a_x = a_x;
    std::vector<Float> w = cola_velocity(p);
    std::memcpy(out, w.data(), 3*np*sizeof(float));
    delete p->pv; free(p->force); delete p;
  });
}

// py_lpt (py/py_lpt.cpp:9-42): 2LPT particles from `seed` with the power
// spectrum table `pk_file`.  The uniform draws come from the stand-in
// stream and are logged (fs2ref_rng_log_*): the first nc^2 fill the seed
// table (py/lpt.cpp:235-273), then column (ix, iy) draws (phase, amplitude)
// for iz = 0 .. nc/2 - 1 (:319-326).
int fs2ref_lpt(int nc, double boxsize, double a, unsigned long seed,
               const char* pk_file, const char* kind, float* x, float* v,
               float* dx1, float* dx2, uint64_t* id) {
  return guarded([&] {
    PowerSpectrum ps(pk_file);
    const size_t nx = fft_local_nx(nc);
    const size_t np_alloc = (size_t)(1.25*(nx + 1)*nc*nc);
    Particles* p = new Particles(np_alloc, boxsize);
    const size_t mem_size = 9*fft_mem_size(nc, 0);
    Mem* const mem = new Mem("LPT", mem_size);
    lpt_init(nc, boxsize, mem);
    lpt_set_displacements(seed, &ps, a, kind, p);
    lpt_free();
    delete mem;
    const size_t np = p->np_local;
    for(size_t i = 0; i < np; i++) {
      for(int k = 0; k < 3; k++) {
        x[3*i + k] = p->p[i].x[k];
        v[3*i + k] = p->p[i].v[k];
        dx1[3*i + k] = p->p[i].dx1[k];
        dx2[3*i + k] = p->p[i].dx2[k];
      }
      id[i] = p->p[i].id;
    }
    delete p->pv; free(p->force); delete p;
  });
}

}  // extern "C"
