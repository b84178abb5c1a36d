/*
 * fs2gpu.h -- C ABI of libfs2gpu.so, the B200 (sm_100a) implementation of
 * fs2's particle-mesh / COLA time step and its 2LPT initial conditions.
 *
 * Each entry point replaces the body of one function of the reference's C++
 * core (LBJ-Wade/fs2, the C++ files under py/) or one method of its CPython
 * extension fs._fs (the py/py_ wrapper files).  The reference function is cited as file:line beside each
 * declaration.  Plain C types only: pointers, sizes, doubles.
 *
 * Conventions
 *  - Every function returns int: FS2G_OK (0) or a negative FS2G_ERR_* code.
 *    The codes mirror the C++ exception classes of py/error.h that the
 *    reference's wrappers turn into Python exceptions (RuntimeError,
 *    AssertionError, IOError, MemoryError) plus FFTError (py/fft.h:185).
 *    fs2g_last_error() returns the message of the last failing call on the
 *    calling thread.  No C++ exception crosses this boundary.
 *  - Device work is ordered on the context's CUDA stream.  Calls that hand
 *    data to the host (the *_copy_out functions, status queries that need a
 *    device value, fs2g_ctx_synchronize) synchronise the stream and report
 *    any error a kernel recorded in the context's device error word (for
 *    example a particle far outside the box) as FS2G_ERR_DEVICE.
 *  - Particle vectors cross the boundary as [n][3] float rows, the layout of
 *    fs.Particles.x (py/py_particles.cpp:306-341); on the device they are
 *    stored as three component planes (structure of arrays).
 *  - A context holds the module state that the reference keeps in file-level
 *    statics (py/pm.cpp:22-30): the PM mesh, its spectrum, FFT plans.  Use one
 *    context per thread or serialise calls on it.
 */
#ifndef FS2GPU_H
#define FS2GPU_H 1

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FS2G_OK              0
#define FS2G_ERR_RUNTIME    (-1)  /* RuntimeError   (py/error.h:10) */
#define FS2G_ERR_ASSERTION  (-2)  /* AssertionError (py/error.h:12) */
#define FS2G_ERR_IO         (-3)  /* IOError        (py/error.h:14) */
#define FS2G_ERR_MEMORY     (-4)  /* MemoryError    (py/error.h:16) */
#define FS2G_ERR_VALUE      (-5)  /* invalid argument (TypeError/ValueError in Python) */
#define FS2G_ERR_FFT        (-6)  /* FFTError       (py/fft.h:185) */
#define FS2G_ERR_CUDA       (-7)  /* CUDA runtime or cuFFT failure */
#define FS2G_ERR_INDEX      (-8)  /* IndexError */
#define FS2G_ERR_DEVICE     (-9)  /* a kernel flagged invalid input */

/* particle fields for copy_in / copy_out / device_field */
#define FS2G_FIELD_X      0   /* Particle::x[3]   (py/particle.h:13) */
#define FS2G_FIELD_V      1   /* Particle::v[3]   (py/particle.h:14) */
#define FS2G_FIELD_DX1    2   /* Particle::dx1[3] (py/particle.h:15) */
#define FS2G_FIELD_DX2    3   /* Particle::dx2[3] (py/particle.h:16) */
#define FS2G_FIELD_FORCE  4   /* Particles::force (py/particle.h:34)  */
#define FS2G_FIELD_ID     5   /* Particle::id, uint64 (py/particle.h:17) */

/* CIC deposit modes (fs2g_pm_set_deposit_mode) */
#define FS2G_DEPOSIT_ATOMIC         0  /* float atomics; summation order varies run to run */
#define FS2G_DEPOSIT_DETERMINISTIC  1  /* sort by cell; fixed-order sums, bitwise reproducible */

/* FFT engine of the PM force (fs2g_pm_set_fft_engine) */
#define FS2G_FFT_AUTO   0  /* the faster engine: the fused pipeline at n = 1024, else cuFFT */
#define FS2G_FFT_CUFFT  1  /* cuFFT R2C, k-space kernel and C2R per axis */
#define FS2G_FFT_FUSED  2  /* fused 5-pass pipeline for n = 64..1024 (powers of 2), else cuFFT */

/* PM status, enum class PmStatus (py/pm.h:8) */
#define FS2G_PM_DENSITY_DONE 0
#define FS2G_PM_FORCE_DONE   1
#define FS2G_PM_DONE         2

typedef struct fs2g_ctx        fs2g_ctx;
typedef struct fs2g_particles  fs2g_particles;
typedef struct fs2g_power      fs2g_power;
typedef struct fs2g_fft        fs2g_fft;

/* ------------------------------------------------------------------ */
/* Library, errors, context                                           */
/* ------------------------------------------------------------------ */
int         fs2g_version(void);
/* message of the last failing call on this thread ("" if none) */
const char* fs2g_last_error(void);

/* Replaces the module-level state of py/pm.cpp:22-30 and the MPI init of
   py/comm.cpp:25-43 (one GPU is one rank). */
int fs2g_ctx_create(int device, fs2g_ctx** out);
int fs2g_ctx_destroy(fs2g_ctx* ctx);
/* run on an external cudaStream_t (e.g. torch's current stream); NULL
   restores the context's own stream */
int fs2g_ctx_set_stream(fs2g_ctx* ctx, void* cuda_stream);
int fs2g_ctx_get_stream(fs2g_ctx* ctx, void** cuda_stream);
int fs2g_ctx_synchronize(fs2g_ctx* ctx);
/* per-stage CUDA-event timing (0 off, 1 on); stages named by
   fs2g_stage_name(i), i < fs2g_stage_count().  Each stage is also an NVTX
   range of that name in the "fs2g" domain, timing on or off, so a profiler
   can select its kernels (ncu --nvtx --nvtx-include "fs2g@deposit/"). */
int fs2g_ctx_set_timing(fs2g_ctx* ctx, int on);
int fs2g_ctx_reset_timing(fs2g_ctx* ctx);
int fs2g_ctx_get_timing(fs2g_ctx* ctx, double* total_ms, long* launches,
                        int nmax);
int         fs2g_stage_count(void);
const char* fs2g_stage_name(int stage);
/* number of kernels this library launched on the context (its own kernels,
   not cuFFT's) since creation */
int fs2g_ctx_kernel_launches(fs2g_ctx* ctx, long* count);

/* ------------------------------------------------------------------ */
/* Cosmology (host FP64), py/cosmology.cpp                            */
/* ------------------------------------------------------------------ */
int fs2g_cosmology_init(double omega_m);                 /* cosmology.cpp:24 */
int fs2g_cosmology_omega_m(double* om);                  /* cosmology.cpp:119 */
int fs2g_cosmology_D_growth(double a, double* D);        /* cosmology.cpp:33 */
int fs2g_cosmology_D2_growth(double a, double D, double* D2); /* :42 */
int fs2g_cosmology_Dv_growth(double a, double D, double* Dv); /* :50 */
int fs2g_cosmology_D2v_growth(double a, double D2, double* D2v); /* :60 */
int fs2g_cosmology_f_growth_rate(double a, double* f);   /* cosmology.cpp:73 */
int fs2g_cosmology_hubble_function(double a, double* H); /* cosmology.cpp:106 */

/* ------------------------------------------------------------------ */
/* Power spectrum table, py/power.cpp                                 */
/* ------------------------------------------------------------------ */
int fs2g_power_alloc(const char* filename, fs2g_power** out); /* power.cpp:15; py_power.cpp:12 */
int fs2g_power_from_table(const double* k, const double* P, int n,
                          fs2g_power** out);
int fs2g_power_free(fs2g_power* ps);                     /* py_power.cpp:42 */
int fs2g_power_n(const fs2g_power* ps, int* n);          /* py_power.cpp:66 */
int fs2g_power_i(const fs2g_power* ps, int i, double* k, double* P); /* py_power.cpp:120 */
int fs2g_power_P(const fs2g_power* ps, double k, double* P); /* power.cpp:50 */
int fs2g_power_sigma(const fs2g_power* ps, double R, double* sigma); /* power.cpp:146 */

/* ------------------------------------------------------------------ */
/* Particles, py/particle.h / py/py_particles.cpp                     */
/* ------------------------------------------------------------------ */
int fs2g_particles_alloc(fs2g_ctx* ctx, size_t np_alloc, double boxsize,
                         fs2g_particles** out);          /* py_particles.cpp:143; particle.cpp:13 */
int fs2g_particles_free(fs2g_particles* p);              /* py_particles.cpp:157 */
int fs2g_particles_len(const fs2g_particles* p, size_t* np_local); /* py_particles.cpp:166 */
int fs2g_particles_np_allocated(const fs2g_particles* p, size_t* n);
int fs2g_particles_np_total(const fs2g_particles* p, uint64_t* n); /* py_particles.cpp:358 */
int fs2g_particles_update_np_total(fs2g_particles* p);   /* particle.cpp:35 */
int fs2g_particles_boxsize(const fs2g_particles* p, double* boxsize);
int fs2g_particles_get_a(const fs2g_particles* p, double* a_x, double* a_v,
                         double* a_f);                   /* Particles::a_x,a_v,a_f */
int fs2g_particles_set_a(fs2g_particles* p, double a_x, double a_v,
                         double a_f);
/* sets np_local (<= np_allocated) */
int fs2g_particles_set_np(fs2g_particles* p, size_t np_local);
/* append n positions from a double array with element strides
   (py_particles.cpp:403-462: only x is written) */
int fs2g_particles_append(fs2g_particles* p, const double* x, size_t n,
                          ptrdiff_t row_stride, ptrdiff_t col_stride);
int fs2g_particles_clear(fs2g_particles* p);             /* py_particles.cpp:386 */
int fs2g_particles_periodic_wrapup(fs2g_particles* p);   /* util.cpp:3 */
/* host <-> device copies of rows [offset, offset+count): vector fields as
   [count][3] float, FS2G_FIELD_ID as uint64 (py_particles.cpp:291-355) */
int fs2g_particles_copy_out(fs2g_particles* p, int field, void* host,
                            size_t offset, size_t count);
int fs2g_particles_copy_in(fs2g_particles* p, int field, const void* host,
                           size_t offset, size_t count);
/* device planes of a field: component c of particle i is at
   ((float*)*dptr)[c*(*plane_stride) + i]; ID is a uint64 array */
int fs2g_particles_device_field(fs2g_particles* p, int field, void** dptr,
                                size_t* plane_stride);
/* v_total = v + Dv dx1 + D2v dx2 at a_x, as [np][3] rows
   (cola_velocity, py/cola.cpp:129-148, with its D1-for-D2 argument) */
int fs2g_cola_velocity(fs2g_ctx* ctx, fs2g_particles* p, float* host);

/* Leapfrog (non-COLA) integrator, py/leapfrog.cpp.
   leapfrog_set_initial_velocity (:18-39): v = dx1 Dv(a) + dx2 D2v(a), a_v = a */
int fs2g_leapfrog_initial_velocity(fs2g_ctx* ctx, fs2g_particles* p, double a);
/* leapfrog_kick (:41-68): v += -1.5 om f Sphi(a_v, a_vel), a_v = a_vel */
int fs2g_leapfrog_kick(fs2g_ctx* ctx, fs2g_particles* p, double a_vel);
/* leapfrog_drift (:70-95): x += v Sq(a_x, a_pos), a_x = a_pos */
int fs2g_leapfrog_drift(fs2g_ctx* ctx, fs2g_particles* p, double a_pos);
/* the kick factor (Float) and dt the calls above would use */
int fs2g_leapfrog_coef(double a_x, double a_v, double a_vel, double a_pos,
                       float* kick_factor, double* dt);

/* ------------------------------------------------------------------ */
/* Particle mesh, py/pm.cpp                                           */
/* ------------------------------------------------------------------ */
int fs2g_pm_init(fs2g_ctx* ctx, int nc_pm, double pm_factor,
                 double boxsize);                        /* pm.cpp:225; py_pm.cpp:10 */
int fs2g_pm_free(fs2g_ctx* ctx);                         /* pm.cpp:270 */
/* periodic wrap of x (pm_domain.cpp:115); the halo exchange of
   pm_domain_send_positions has no counterpart on one GPU */
int fs2g_pm_send_positions(fs2g_ctx* ctx, fs2g_particles* p); /* pm_domain.cpp:94; py_pm.cpp:88 */
int fs2g_pm_compute_density(fs2g_ctx* ctx, fs2g_particles* p); /* pm.cpp:341; py_pm.cpp:34 */
/* <delta> = 0 check; a no-op unless fs2g_pm_set_check(ctx, 1), as the
   reference's is a no-op unless built with -DCHECK */
int fs2g_pm_check_total_density(fs2g_ctx* ctx);          /* pm.cpp:357; py_pm.cpp:113 */
int fs2g_pm_compute_force(fs2g_ctx* ctx, fs2g_particles* p); /* pm.cpp:306; py_pm.cpp:59 */
int fs2g_pm_get_forces(fs2g_ctx* ctx, fs2g_particles* p); /* pm_domain.cpp:129 (no-op) */
/* fs.pm.force (py/fs/pm.py:17-31): send_positions, compute_density,
   check_total_density, compute_force, get_forces */
int fs2g_pm_force(fs2g_ctx* ctx, fs2g_particles* p);
int fs2g_pm_set_deposit_mode(fs2g_ctx* ctx, int mode);
/* The deterministic deposit's tile (bin) shape: shape in
   0 .. FS2G_BIN_SHAPES - 1 fixes it (0: 16 x 16 x 32 cells, 1: 16 x 8 x 32,
   2: 8 x 8 x 32, 3: 8 x 8 x 16, 4: 4 x 4 x 32); -1 (the default) lets the
   autotuner time every shape at the first deterministic deposit of each
   (mesh, particle count) and keep the fastest.  The density is the same,
   bit for bit, with every shape.  No reference counterpart. */
#define FS2G_BIN_SHAPES 5
int fs2g_pm_set_bin_tile(fs2g_ctx* ctx, int shape);
/* the shape the last deterministic deposit used (-1 before the first):
   its index and sides in cells */
int fs2g_pm_get_bin_tile(fs2g_ctx* ctx, int* shape, int* tx, int* ty,
                         int* tz);
/* how the last deterministic deposit binned its particles (waits for it):
   1 one pass into bins sized from the previous deposit's counts (entries
   beyond a bin's room binned from an overflow list), 2 the two passes
   (count, scatter), 3 one pass whose overflow list filled up, followed by
   the two-pass scatter; 0 before the first */
int fs2g_pm_get_bin_pass(fs2g_ctx* ctx, int* passes);
int fs2g_pm_set_check(fs2g_ctx* ctx, int on);
/* choose the FFT engine; takes effect at the next fs2g_pm_init with new
   arguments or after fs2g_pm_free */
int fs2g_pm_set_fft_engine(fs2g_ctx* ctx, int engine);
/* keep delta(k) in HBM during compute_force so that
   fs2g_pm_delta_k_copy_out can return it (the fused engine otherwise never
   writes it) */
int fs2g_pm_set_keep_delta_k(fs2g_ctx* ctx, int on);
int fs2g_pm_fft_engine(fs2g_ctx* ctx, int* fused);
/* kz columns per tile of the fused pipeline's y and x passes (4 or 8; a
   tuning parameter, results are identical) */
int fs2g_pm_set_fft_tile(fs2g_ctx* ctx, int columns);
int fs2g_pm_status(fs2g_ctx* ctx, int* status);          /* pm.cpp:398 */
int fs2g_pm_nc(fs2g_ctx* ctx, int* nc);
/* the PM mesh as an FFT handle (non-owning), the "_FFT" capsule that
   _pm_compute_density returns (py_pm.cpp:53-55).  After a density it
   holds the density contrast.  After a force its copy-out returns the z
   force component, as the reference's in-place buffer does.  The fused
   n = 1024 pipeline has by then reset the density mesh itself to -1 for
   the next deposit. */
int fs2g_pm_fft(fs2g_ctx* ctx, fs2g_fft** out);
/* unnormalised delta(k), [n][n][n/2+1] complex as float pairs */
int fs2g_pm_delta_k_copy_out(fs2g_ctx* ctx, float* host);
/* force mesh of one axis, [n][n][n] float (after compute_force) */
int fs2g_pm_force_mesh_copy_out(fs2g_ctx* ctx, int axis, float* host);

/* ------------------------------------------------------------------ */
/* COLA, py/cola.cpp                                                  */
/* ------------------------------------------------------------------ */
int fs2g_cola_kick(fs2g_ctx* ctx, fs2g_particles* p, double a_vel);  /* cola.cpp:48; py_cola.cpp:4 */
int fs2g_cola_drift(fs2g_ctx* ctx, fs2g_particles* p, double a_pos); /* cola.cpp:94; py_cola.cpp:24 */
/* kick to a_vel then drift to a_pos in one pass over the particles;
   the same arithmetic as fs2g_cola_kick followed by fs2g_cola_drift */
int fs2g_cola_kick_drift(fs2g_ctx* ctx, fs2g_particles* p, double a_vel,
                         double a_pos);
/* the host FP64 coefficients of the two loops: kick from a_v to a_vel with
   the force at a_x (py/cola.cpp:50-66), drift from a_x to a_pos with
   velocities at a_v (py/cola.cpp:96-109, Sq at :152-179) */
int fs2g_cola_kick_coef(double a_v, double a_x, double a_vel, double* neg15om,
                        float* kick_factor, float* q1, float* q2);
int fs2g_cola_drift_coef(double a_x, double a_v, double a_pos, double* dt,
                         float* da1, float* da2);
/* one step of the time loop of script/cola.py:37-44: force at a_x, kick to
   a_vel, drift to a_pos */
int fs2g_cola_step(fs2g_ctx* ctx, fs2g_particles* p, double a_vel,
                   double a_pos);

/* ------------------------------------------------------------------ */
/* 2LPT initial conditions, py/lpt.cpp                                */
/* ------------------------------------------------------------------ */
/* fs._fs._lpt (py_lpt.cpp:9-42): kind is "zeldovich", "2lpt" or "cola".
   The Gaussian field's uniform draws come from this library's counter-based
   generator keyed by (seed, kx, ky, iz); they are not GSL ranlxd1's. */
int fs2g_lpt(fs2g_ctx* ctx, int nc, double boxsize, double a,
             unsigned long seed, const fs2g_power* ps, const char* kind,
             fs2g_particles** out);
/* the same with the draws of py/lpt.cpp:322-326 given: u_phase and u_ampl
   are [nc][nc][nc/2] doubles in (0,1] (column-major in iz) */
int fs2g_lpt_from_draws(fs2g_ctx* ctx, int nc, double boxsize, double a,
                        const double* u_phase, const double* u_ampl,
                        const fs2g_power* ps, const char* kind,
                        fs2g_particles** out);
/* the same from a given unnormalised delta(k), [nc][nc][nc/2+1] complex
   float pairs (e.g. a white-noise field); Nyquist planes and k=0 are
   dropped as lpt_generate_psi_k leaves them (py/lpt.cpp:328-331) */
int fs2g_lpt_from_delta_k(fs2g_ctx* ctx, int nc, double boxsize, double a,
                          const float* delta_k, const char* kind,
                          fs2g_particles** out);
/* the generator's draws for (nc, seed), same layout as above */
int fs2g_lpt_draws(fs2g_ctx* ctx, int nc, unsigned long seed,
                   double* u_phase, double* u_ampl);
int fs2g_lpt_set_offset(double offset);                  /* lpt.cpp:227 */
int fs2g_lpt_set_zeldovich_force(fs2g_ctx* ctx, fs2g_particles* p,
                                 double a);              /* py_lpt.cpp:57 */

/* ------------------------------------------------------------------ */
/* FFT mesh objects, py/fft.cpp / py/py_fft.cpp                       */
/* ------------------------------------------------------------------ */
int fs2g_fft_alloc(fs2g_ctx* ctx, int nc, fs2g_fft** out); /* py_fft.cpp:28 */
int fs2g_fft_free(fs2g_fft* fft);                        /* py_fft.cpp:48 (no-op on the PM mesh) */
int fs2g_fft_nc(const fs2g_fft* fft, int* nc);
int fs2g_fft_set_test_data(fs2g_fft* fft);               /* py_fft.cpp:57 */
/* the real mesh as [nc][nc][nc] float (py_fft.cpp:87-188) */
int fs2g_fft_fx_copy_out(fs2g_fft* fft, float* host);

/* ------------------------------------------------------------------ */
/* Differentiable COLA (no counterpart in the reference)              */
/* ------------------------------------------------------------------ */
/* A simulation from a white-noise field w (nc^3 reals, dense [x][y][z]):
   delta(k) = T(k) FFT(w), T = sqrt(P(k)/(V nc^3)) with k = 0 and the
   Nyquist planes dropped; 2LPT particles at a_init ('cola' kind); nsteps
   COLA steps with the given (a_vel, a_pos) schedule on an n^3 PM mesh; the
   CIC density contrast of the final positions (n^3 reals, dense).  The
   backward maps a cotangent of that density to dL/dw with hand-written
   adjoints of every stage, recomputing each step's meshes from per-step
   checkpoints of (x, v).  The run uses the context's PM module (it calls
   fs2g_pm_init(ctx, n, n/nc, boxsize)).  All array arguments of forward and
   backward are device pointers. */
typedef struct fs2g_diff fs2g_diff;
int fs2g_diff_create(fs2g_ctx* ctx, int nc, int n, double boxsize,
                     const fs2g_power* ps, double a_init, int nsteps,
                     const double* a_vel, const double* a_pos,
                     fs2g_diff** out);
int fs2g_diff_free(fs2g_diff* d);
int fs2g_diff_forward(fs2g_diff* d, const float* white_noise,
                      float* delta_out);
int fs2g_diff_backward(fs2g_diff* d, const float* delta_bar,
                       float* white_noise_bar);
/* the simulation's particles (final state after forward) */
int fs2g_diff_particles(fs2g_diff* d, fs2g_particles** p);

/* ------------------------------------------------------------------ */
/* Ensemble of differentiable runs of uneven sizes.  No counterpart in  */
/* the reference (its scripts loop over realisations, one MPI job each). */
/* Member i is a differentiable run (nc[i] particles per side, an n[i]  */
/* mesh, box boxsize[i]) with device buffers for its white noise        */
/* (nc^3), target and density (n^3) and gradient (nc^3).  A run         */
/* computes, per member: density = forward(noise), loss =               */
/* mean((density - target)^2), gradient = d loss / d noise.             */
/* Members of one (nc, n, boxsize) form a size class, run in chunks:    */
/* each chunk is one batched run whose every kernel and (batched cuFFT) */
/* transform covers all of the chunk's members.                         */
/* FS2G_ENSEMBLE_GRAPH forks the chunks onto their own streams,          */
/* captured once into a CUDA graph and replayed with one launch;         */
/* FS2G_ENSEMBLE_LOOP runs each member alone through the unbatched path, */
/* one after another on the stream of `ctx`.                             */
/* autotune != 0: per size class, time forward + loss + backward with    */
/* B, B/2 and B/4 members per chunk and keep the fastest (else B).       */
/* Members take ctx's deposit mode at creation.                         */
/* ------------------------------------------------------------------ */
typedef struct fs2g_ensemble fs2g_ensemble;
#define FS2G_ENSEMBLE_LOOP  0
#define FS2G_ENSEMBLE_GRAPH 1
int fs2g_ensemble_create(fs2g_ctx* ctx, int count, const int* nc,
                         const int* n, const double* boxsize,
                         const fs2g_power* ps, double a_init, int nsteps,
                         const double* a_vel, const double* a_pos,
                         int autotune, fs2g_ensemble** out);
int fs2g_ensemble_free(fs2g_ensemble* e);
int fs2g_ensemble_size(const fs2g_ensemble* e, int* count);
/* device buffers of member i (any pointer may be NULL) */
int fs2g_ensemble_member(fs2g_ensemble* e, int i, float** white_noise,
                         float** target, float** density, float** gradient,
                         int* nc, int* n);
/* the choice for member i's size class: FS2G_FFT_* engine, members per
   chunk, and the class's forward + loss + backward time the autotuner
   measured with it (ms; 0 when not tuned) */
int fs2g_ensemble_tuning(const fs2g_ensemble* e, int i, int* engine,
                         int* chunk, double* ms);
/* forward only of member i into its density buffer (synchronous) */
int fs2g_ensemble_forward_member(fs2g_ensemble* e, int i);
/* one run of every member (asynchronous on ctx's stream) */
int fs2g_ensemble_run(fs2g_ensemble* e, int mode);
/* waits for the last run; host[i] = member i's loss */
int fs2g_ensemble_losses(fs2g_ensemble* e, double* host);
/* kernel launches in one graph replay (0 before the first graph run) */
int fs2g_ensemble_graph_kernels(const fs2g_ensemble* e, long* count);

/* ------------------------------------------------------------------ */
/* Allocation-free CIC density                                        */
/* ------------------------------------------------------------------ */
/* No counterpart in the reference.  For callers that may not have the
   library allocate device memory mid-run: those that own all device memory
   themselves (an up-front arena, a framework's caching allocator), and those
   calling from a time loop that cannot absorb cudaFree's device-wide
   synchronisation.  Writes the deterministic CIC density contrast of np
   particles -- -1 plus the binned fixed-point deposit, bit for bit the
   result of fs2g_pm_compute_density in FS2G_DEPOSIT_DETERMINISTIC mode --
   into `mesh`, a device array [n][n][2(n/2+1)] floats (every cell with
   iz < n is written; the row padding is not touched).  x0, x1, x2 are device
   arrays of the three position components, wrapped into [0, boxsize).  It
   calls no cudaMalloc, cudaFree or allocating library routine: its scratch
   is one file-scope device array of FS2G_NOALLOC_SCRATCH_BYTES that every
   GPU which loads the library keeps until the process exits, so np is
   limited to FS2G_NOALLOC_MAX_PARTICLES and n to FS2G_NOALLOC_MAX_MESH
   (beyond either it returns FS2G_ERR_VALUE).  A device's first call (and
   the first after a new CUDA context replaces the old one on that device,
   e.g. after cudaDeviceReset) looks up the array's device address with that
   device current.  The call synchronises `cuda_stream` (NULL: the legacy
   default stream) and reads back an error word, so it must not be made
   while any stream is being captured into a CUDA graph.  All calls share the
   one array and each zeroes the parts that must start at zero: calls that
   overlap on the GPU (other streams, other host threads) race and must be
   serialised by the caller. */
#define FS2G_NOALLOC_MAX_PARTICLES 262144
#define FS2G_NOALLOC_MAX_MESH 1024
#define FS2G_NOALLOC_SCRATCH_BYTES 10486016
int fs2g_cic_density_noalloc(const float* x0, const float* x1, const float* x2,
                             size_t np, float* mesh, int n, double boxsize,
                             double pm_factor, void* cuda_stream);

#ifdef __cplusplus
}
#endif

#endif
