/*
 * fs2_oracle.c -- CPU restatement of fs2's particle-mesh / COLA / 2LPT loops.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA path is
 * compared against; the product never links, loads or calls it.  It is also
 * timed, with OpenMP, as the CPU baseline beside the GPU numbers.
 *
 * Every function restates one loop of the reference (LBJ-Wade/fs2, C++11
 * core under py/) with the same evaluation order and the same float/double
 * promotions, so that a serial (1-thread) run reproduces the reference's
 * serial arithmetic.  Build with -ffp-contract=off: the reference is built
 * for plain x86-64 (SSE2, no FMA), so no product is fused into an add.
 *
 * Data layout is the reference's own: positions and the other particle
 * vectors are [np][3] float rows (as fs.Particles.x returns them), the real
 * mesh is [n][n][ncz] floats with ncz = 2(n/2+1) (py/pm.cpp:242), and the
 * complex half spectrum is [n][n][n/2+1] (float re, float im) pairs.  The
 * reference stores the PM spectrum transposed ([ky][kx][kz],
 * FFTW_MPI_TRANSPOSED_OUT, py/fft.cpp:53); the value at each (kx,ky,kz) is the
 * same, only the storage order differs, and this file uses [kx][ky][kz].
 *
 * Parity pins: the single-particle CIC cases of test/test_pm_cic.py, the
 * sum(delta)=0 invariant of test/test_pm_density.py, the a=0 grid and ids of
 * test/test_particles_h5.py and the mesh layout of test/test_fft.py are
 * checked in tests/test_oracle.py.  The reference ships no golden output
 * files (test/.gitignore ignores *.h5), so there is nothing else to pin to.
 */
#include <stddef.h>
#include <stdint.h>
#include <math.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef M_PI
#define M_PI 3.14159265358979323846264338327950288
#endif

typedef float Float;

static inline size_t mesh_index(size_t ix, size_t iy, size_t iz,
                                size_t nc, size_t ncz)
{
  /* grid_assign / grid_val index, py/pm.cpp:38,44 */
  return (ix*nc + iy)*ncz + iz;
}

static void set_threads(int nthreads)
{
#ifdef _OPENMP
  if(nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void) nthreads;
#endif
}

/* ------------------------------------------------------------------ */
/* periodic wrap: periodic_wrapup_p, py/util.h:14-24 (single fold)     */
/* ------------------------------------------------------------------ */
void or_periodic_wrap(Float* x, size_t np, Float boxsize)
{
  for(size_t i=0; i<np; i++) {
    for(int k=0; k<3; k++) {
      Float v= x[3*i + k];
      if(v < 0) v += boxsize;
      if(v >= boxsize) v -= boxsize;
      x[3*i + k]= v;
    }
  }
}

/* ------------------------------------------------------------------ */
/* clear_density, py/pm.cpp:414-426: mesh = -1 for iz < n only         */
/* ------------------------------------------------------------------ */
void or_clear_density(Float* mesh, int nc_)
{
  const size_t nc= (size_t) nc_;
  const size_t ncz= 2*(nc/2 + 1);
  for(size_t ix=0; ix<nc; ix++)
    for(size_t iy=0; iy<nc; iy++)
      for(size_t iz=0; iz<nc; iz++)
        mesh[mesh_index(ix, iy, iz, nc, ncz)]= -1;
}

/* CIC cell indices and weights, shared by deposit and gather.
   py/pm.cpp:85-115 (deposit) and :156-192 (gather) compute them the same
   way: X = x*dx_inv in Float, (int) truncation, w1 = X - i0, w0 = 1 - w1,
   i0 >= n -> 0 (after the weights), i1 = i0 + 1 wrapped. */
typedef struct {
  int i0[3], i1[3];
  Float w0[3], w1[3];
} cic_t;

static inline void cic_setup(const Float* xp, Float dx_inv, int nci, cic_t* c)
{
  for(int k=0; k<3; k++) {
    Float X= xp[k]*dx_inv;
    int i0= (int) X;
    Float w1= X - i0;
    Float w0= 1 - w1;
    if(i0 >= nci) i0= 0;
    int i1= i0 + 1; if(i1 >= nci) i1 -= nci;
    c->i0[k]= i0; c->i1[k]= i1;
    c->w0[k]= w0; c->w1[k]= w1;
  }
}

/* ------------------------------------------------------------------ */
/* pm_assign_cic_density<Particle>, py/pm.cpp:57-139                   */
/* nthreads <= 1: serial particle order (the reference's serial run). */
/* nthreads > 1: OpenMP with atomic adds, as py/pm.cpp:35-37,81-83.   */
/* ------------------------------------------------------------------ */
void or_cic_deposit(const Float* x, size_t np, Float* mesh, int nc_,
                    Float boxsize, double pm_factor, int nthreads)
{
  const size_t nc= (size_t) nc_;
  const size_t ncz= 2*(nc/2 + 1);
  const Float dx_inv= nc/boxsize;                    /* py/pm.cpp:77 */
  const Float fac= pm_factor*pm_factor*pm_factor;    /* py/pm.cpp:78 */
  const int nci= nc_;

  if(nthreads <= 1) {
    for(size_t i=0; i<np; i++) {
      cic_t c; cic_setup(x + 3*i, dx_inv, nci, &c);
      const size_t ix0= c.i0[0], iy0= c.i0[1], iz0= c.i0[2];
      const size_t ix1= c.i1[0], iy1= c.i1[1], iz1= c.i1[2];
      const Float wx0= c.w0[0], wy0= c.w0[1], wz0= c.w0[2];
      const Float wx1= c.w1[0], wy1= c.w1[1], wz1= c.w1[2];
      mesh[mesh_index(ix0, iy0, iz0, nc, ncz)] += fac*wx0*wy0*wz0;
      mesh[mesh_index(ix0, iy0, iz1, nc, ncz)] += fac*wx0*wy0*wz1;
      mesh[mesh_index(ix0, iy1, iz0, nc, ncz)] += fac*wx0*wy1*wz0;
      mesh[mesh_index(ix0, iy1, iz1, nc, ncz)] += fac*wx0*wy1*wz1;
      mesh[mesh_index(ix1, iy0, iz0, nc, ncz)] += fac*wx1*wy0*wz0;
      mesh[mesh_index(ix1, iy0, iz1, nc, ncz)] += fac*wx1*wy0*wz1;
      mesh[mesh_index(ix1, iy1, iz0, nc, ncz)] += fac*wx1*wy1*wz0;
      mesh[mesh_index(ix1, iy1, iz1, nc, ncz)] += fac*wx1*wy1*wz1;
    }
    return;
  }

  set_threads(nthreads);
#pragma omp parallel for schedule(static)
  for(size_t i=0; i<np; i++) {
    cic_t c; cic_setup(x + 3*i, dx_inv, nci, &c);
    const size_t ix0= c.i0[0], iy0= c.i0[1], iz0= c.i0[2];
    const size_t ix1= c.i1[0], iy1= c.i1[1], iz1= c.i1[2];
    const Float wx0= c.w0[0], wy0= c.w0[1], wz0= c.w0[2];
    const Float wx1= c.w1[0], wy1= c.w1[1], wz1= c.w1[2];
    Float v;
#define OR_ADD(ix, iy, iz, w) \
    v= (w); \
    _Pragma("omp atomic") \
    mesh[mesh_index(ix, iy, iz, nc, ncz)] += v;
    OR_ADD(ix0, iy0, iz0, fac*wx0*wy0*wz0)
    OR_ADD(ix0, iy0, iz1, fac*wx0*wy0*wz1)
    OR_ADD(ix0, iy1, iz0, fac*wx0*wy1*wz0)
    OR_ADD(ix0, iy1, iz1, fac*wx0*wy1*wz1)
    OR_ADD(ix1, iy0, iz0, fac*wx1*wy0*wz0)
    OR_ADD(ix1, iy0, iz1, fac*wx1*wy0*wz1)
    OR_ADD(ix1, iy1, iz0, fac*wx1*wy1*wz0)
    OR_ADD(ix1, iy1, iz1, fac*wx1*wy1*wz1)
#undef OR_ADD
  }
}

/* ------------------------------------------------------------------ */
/* force_at_particle_locations<Particle>, py/pm.cpp:142-220            */
/* f is [np][3]; only component `axis` is written.                     */
/* ------------------------------------------------------------------ */
void or_force_gather(const Float* x, size_t np, const Float* fx, int nc_,
                     Float boxsize, int axis, Float* f, int nthreads)
{
  const size_t nc= (size_t) nc_;
  const size_t ncz= 2*(nc/2 + 1);
  const Float dx_inv= nc/boxsize;                    /* py/pm.cpp:146 */
  const int nci= nc_;

  set_threads(nthreads);
#pragma omp parallel for schedule(static) if(nthreads > 1)
  for(size_t i=0; i<np; i++) {
    cic_t c; cic_setup(x + 3*i, dx_inv, nci, &c);
    const size_t ix0= c.i0[0], iy0= c.i0[1], iz0= c.i0[2];
    const size_t ix1= c.i1[0], iy1= c.i1[1], iz1= c.i1[2];
    const Float wx0= c.w0[0], wy0= c.w0[1], wz0= c.w0[2];
    const Float wx1= c.w1[0], wy1= c.w1[1], wz1= c.w1[2];

    Float fi= 0;                                     /* py/pm.cpp:203 */
    fi += fx[mesh_index(ix0, iy0, iz0, nc, ncz)]*wx0*wy0*wz0 +
          fx[mesh_index(ix0, iy0, iz1, nc, ncz)]*wx0*wy0*wz1 +
          fx[mesh_index(ix0, iy1, iz0, nc, ncz)]*wx0*wy1*wz0 +
          fx[mesh_index(ix0, iy1, iz1, nc, ncz)]*wx0*wy1*wz1;
    fi += fx[mesh_index(ix1, iy0, iz0, nc, ncz)]*wx1*wy0*wz0 +
          fx[mesh_index(ix1, iy0, iz1, nc, ncz)]*wx1*wy0*wz1 +
          fx[mesh_index(ix1, iy1, iz0, nc, ncz)]*wx1*wy1*wz0 +
          fx[mesh_index(ix1, iy1, iz1, nc, ncz)]*wx1*wy1*wz1;
    f[3*i + axis]= fi;
  }
}

/* ------------------------------------------------------------------ */
/* compute_force_mesh(axis) k-space part, py/pm.cpp:460-505            */
/* delta_k, fk: [n][n][n/2+1] complex as interleaved floats.           */
/* ------------------------------------------------------------------ */
void or_force_mesh_k(const Float* delta_k, Float* fk, int nc_, Float boxsize,
                     int axis, int nthreads)
{
  const size_t nc= (size_t) nc_;
  const size_t nckz= nc/2 + 1;
  const int nci= nc_;
  const Float f1= -1.0/pow(nc, 3.0)/(2.0*M_PI/boxsize);   /* py/pm.cpp:472 */

  fk[0]= 0; fk[1]= 0;                                      /* py/pm.cpp:469 */

  set_threads(nthreads);
#pragma omp parallel for schedule(static) if(nthreads > 1)
  for(size_t iy=0; iy<nc; iy++) {
    int iy0= (int) iy <= (nci/2) ? (int) iy : (int) iy - nci;   /* :483 */
    Float k[3];
    k[1]= (Float) iy0;
    for(size_t ix=0; ix<nc; ix++) {
      int ix0= ix <= (nc/2) ? (int) ix : (int) ix - nci;       /* :489 */
      k[0]= (Float) ix0;
      size_t kzmin= (ix == 0 && iy == 0);                      /* :492 */
      for(size_t iz=kzmin; iz<nckz; iz++) {
        k[2]= (Float) iz;
        Float f2= f1/(k[0]*k[0] + k[1]*k[1] + k[2]*k[2])*k[axis];
        size_t index= (nc*ix + iy)*nckz + iz;
        fk[2*index    ]= -f2*delta_k[2*index + 1];
        fk[2*index + 1]=  f2*delta_k[2*index    ];
      }
    }
  }
}

/* ------------------------------------------------------------------ */
/* cola_kick particle loop, py/cola.cpp:79-88.  The host computes      */
/* kick_factor and q1, q2 as Float and om in double (:57-66); the      */
/* product with -1.5*om is evaluated in double then rounded.           */
/* ------------------------------------------------------------------ */
void or_cola_kick(const Float* f, const Float* dx1, const Float* dx2,
                  Float* v, size_t np, double om, Float kick_factor,
                  Float q1, Float q2, int nthreads)
{
  set_threads(nthreads);
#pragma omp parallel for schedule(static) if(nthreads > 1)
  for(size_t i=0; i<np; i++) {
    for(int k=0; k<3; k++) {
      Float a= -1.5*om*(f[3*i+k] + dx1[3*i+k]*q1 + dx2[3*i+k]*q2);
      v[3*i+k] += a*kick_factor;
    }
  }
}

/* ------------------------------------------------------------------ */
/* cola_drift particle loop, py/cola.cpp:117-124.  v*dt is a double    */
/* product, the displacement bracket is float, the sum is double.      */
/* ------------------------------------------------------------------ */
void or_cola_drift(Float* x, const Float* v, const Float* dx1,
                   const Float* dx2, size_t np, double dt, Float da1,
                   Float da2, int nthreads)
{
  set_threads(nthreads);
#pragma omp parallel for schedule(static) if(nthreads > 1)
  for(size_t i=0; i<np; i++) {
    for(int k=0; k<3; k++) {
      x[3*i+k] += v[3*i+k]*dt + (dx1[3*i+k]*da1 + dx2[3*i+k]*da2);
    }
  }
}

/* ------------------------------------------------------------------ */
/* Leapfrog (non-COLA) particle loops, py/leapfrog.cpp:18-95.           */
/* Initial velocity in float; the kick's -1.5*om*f*kick_factor and the  */
/* drift's v*dt are double products added to the float in double.       */
/* ------------------------------------------------------------------ */
void or_leapfrog_velocity(const Float* dx1, const Float* dx2, Float* v,
                          size_t np, Float Dv, Float D2v)
{
  for(size_t i=0; i<3*np; i++)
    v[i]= dx1[i]*Dv + dx2[i]*D2v;
}

void or_leapfrog_kick(const Float* f, Float* v, size_t np, double om,
                      Float kick_factor)
{
  for(size_t i=0; i<3*np; i++)
    v[i] += -1.5*om*f[i]*kick_factor;
}

void or_leapfrog_drift(Float* x, const Float* v, size_t np, double dt)
{
  for(size_t i=0; i<3*np; i++)
    x[i] += v[i]*dt;
}

/* ================================================================== */
/* 2LPT                                                                */
/* ================================================================== */

/* Natural cubic spline of ln P(ln k), evaluated as
   c3*t^3 + c2*t^2 + c1*t + c0 with t = ln k - knot[j] on [knot[j],knot[j+1]).
   The coefficients come from the caller (scipy CubicSpline, natural end
   conditions), which restates gsl_interp_cspline of py/power.cpp:31-55. */
typedef struct {
  const double* knots;   /* n */
  const double* coef;    /* 4 x (n-1), row-major: c3, c2, c1, c0 */
  int n;
} or_spline_t;

static double spline_P(const or_spline_t* s, double k)
{
  const double lk= log(k);
  int lo= 0, hi= s->n - 1;
  if(lk <= s->knots[0]) lo= 0;
  else if(lk >= s->knots[hi]) lo= hi - 1;
  else {
    while(hi - lo > 1) {
      int mid= (lo + hi)/2;
      if(s->knots[mid] > lk) hi= mid; else lo= mid;
    }
  }
  const int m= s->n - 1;
  const double t= lk - s->knots[lo];
  const double c3= s->coef[0*m + lo], c2= s->coef[1*m + lo];
  const double c1= s->coef[2*m + lo], c0= s->coef[3*m + lo];
  return exp(((c3*t + c2)*t + c1)*t + c0);
}

/* ------------------------------------------------------------------ */
/* lpt_generate_psi_k, py/lpt.cpp:276-436 (single rank: local_ix0 = 0, */
/* local_nx = nc).  The GSL draws of :322-326 are inputs here:         */
/* u_phase[ix][iy][iz] and u_ampl[ix][iy][iz] for iz < nc/2, in (0,1). */
/* psi_k: 3 arrays [nc][nc][nc/2+1] complex.                           */
/* ------------------------------------------------------------------ */
void or_lpt_psi_k(int nc_, double boxsize, const double* u_phase,
                  const double* u_ampl, const double* knots,
                  const double* coef, int nknots, Float* psi_k0,
                  Float* psi_k1, Float* psi_k2)
{
  const size_t nc= (size_t) nc_;
  const size_t nckz= nc/2 + 1;
  const size_t nzd= nc/2;                   /* draws per column */
  const double dk= 2.0*M_PI/boxsize;
  const double knq= nc*M_PI/boxsize;
  const double fac= pow(2*M_PI/boxsize, 1.5);
  const double fac_2pi3= 1.0/(8.0*M_PI*M_PI*M_PI);
  Float* psi_k[3]= {psi_k0, psi_k1, psi_k2};
  or_spline_t ps= {knots, coef, nknots};

  for(size_t i=0; i<nc*nc*nckz*2; i++)      /* :299-306 */
    psi_k0[i]= psi_k1[i]= psi_k2[i]= 0;

  double kvec[3];
  for(size_t ix=0; ix<nc; ix++) {
    for(size_t iy=0; iy<nc; iy++) {
      for(size_t iz=0; iz<nc/2; iz++) {
        const size_t d= (ix*nc + iy)*nzd + iz;
        double phase= u_phase[d]*2*M_PI;           /* :322 */
        double ampl= u_ampl[d];                    /* :324-326 */

        if(ix == nc/2 || iy == nc/2 || iz == nc/2) /* :328 */
          continue;
        if(ix == 0 && iy == 0 && iz == 0)
          continue;

        if(ix < nc/2) kvec[0]= dk*ix; else kvec[0]= -dk*(nc - ix);
        if(iy < nc/2) kvec[1]= dk*iy; else kvec[1]= -dk*(nc - iy);
        if(iz < nc/2) kvec[2]= dk*iz; else kvec[2]= -dk*(nc - iz);

        double kmag2= kvec[0]*kvec[0] + kvec[1]*kvec[1] + kvec[2]*kvec[2];
        double kmag= sqrt(kmag2);

        if(fabs(kvec[0]) > knq) continue;          /* :356-361 */
        if(fabs(kvec[1]) > knq) continue;
        if(fabs(kvec[2]) > knq) continue;

        double delta2= -log(ampl)*fac_2pi3*spline_P(&ps, kmag);
        double delta_k_mag= fac*sqrt(delta2);

        if(iz > 0) {                                /* :370-378 */
          size_t index= (ix*nc + iy)*nckz + iz;
          for(int i=0; i<3; i++) {
            psi_k[i][2*index    ]= -kvec[i]/kmag2*delta_k_mag*sin(phase);
            psi_k[i][2*index + 1]=  kvec[i]/kmag2*delta_k_mag*cos(phase);
          }
        }
        else {                                      /* :379-426 */
          if(ix == 0) {
            if(iy >= nc/2)
              continue;
            size_t iiy= nc - iy;
            size_t index= (ix*nc + iy)*nckz + iz;
            size_t iindex= (ix*nc + iiy)*nckz + iz;
            for(int i=0; i<3; i++) {
              psi_k[i][2*index    ]= -kvec[i]/kmag2*delta_k_mag*sin(phase);
              psi_k[i][2*index + 1]=  kvec[i]/kmag2*delta_k_mag*cos(phase);
              psi_k[i][2*iindex    ]= -kvec[i]/kmag2*delta_k_mag*sin(phase);
              psi_k[i][2*iindex + 1]= -kvec[i]/kmag2*delta_k_mag*cos(phase);
            }
          }
          else {
            if(ix >= nc/2)
              continue;
            size_t iix= nc - ix;
            if(iix == nc) iix= 0;
            size_t iiy= nc - iy;
            if(iiy == nc) iiy= 0;
            size_t index= (ix*nc + iy)*nckz + iz;
            for(int i=0; i<3; i++) {
              psi_k[i][2*index    ]= -kvec[i]/kmag2*delta_k_mag*sin(phase);
              psi_k[i][2*index + 1]=  kvec[i]/kmag2*delta_k_mag*cos(phase);
            }
            index= (iix*nc + iiy)*nckz + iz;
            for(int i=0; i<3; i++) {
              psi_k[i][2*index    ]= -kvec[i]/kmag2*delta_k_mag*sin(phase);
              psi_k[i][2*index + 1]= -kvec[i]/kmag2*delta_k_mag*cos(phase);
            }
          }
        }
      }
    }
  }
}

/* LPT wavenumber for index i, py/lpt.cpp:469-482 (Nyquist -> negative) */
static inline double lpt_k(size_t i, size_t nc, double dk)
{
  return i < nc/2 ? dk*i : -dk*(nc - i);
}

/* ------------------------------------------------------------------ */
/* lpt_compute_psi2_k first loop, py/lpt.cpp:465-505:                  */
/* psi_ij(k) = i k_j psi_i(k) for (11,12,13,22,23,33).                 */
/* ------------------------------------------------------------------ */
void or_lpt_psi_ij_k(int nc_, double boxsize, const Float* psi_k0,
                     const Float* psi_k1, const Float* psi_k2,
                     Float* out0, Float* out1, Float* out2,
                     Float* out3, Float* out4, Float* out5)
{
  const size_t nc= (size_t) nc_;
  const size_t nckz= nc/2 + 1;
  const double dk= 2.0*M_PI/boxsize;
  const Float* psi_k[3]= {psi_k0, psi_k1, psi_k2};
  Float* o[6]= {out0, out1, out2, out3, out4, out5};
  /* (component i, derivative j) for the six outputs */
  static const int ci[6]= {0, 0, 0, 1, 1, 2};
  static const int cj[6]= {0, 1, 2, 1, 2, 2};

  for(size_t ix=0; ix<nc; ix++) {
    for(size_t iy=0; iy<nc; iy++) {
      for(size_t iz=0; iz<nckz; iz++) {
        size_t index= (ix*nc + iy)*nckz + iz;
        double kvec[3]= {lpt_k(ix, nc, dk), lpt_k(iy, nc, dk),
                         lpt_k(iz, nc, dk)};
        for(int m=0; m<6; m++) {
          const Float* p= psi_k[ci[m]];
          o[m][2*index    ]= -p[2*index + 1]*kvec[cj[m]];
          o[m][2*index + 1]=  p[2*index    ]*kvec[cj[m]];
        }
      }
    }
  }
}

/* ------------------------------------------------------------------ */
/* 2LPT source in real space, py/lpt.cpp:522-535 (padded meshes).      */
/* ------------------------------------------------------------------ */
void or_lpt_source(int nc_, const Float* p0, const Float* p1, const Float* p2,
                   const Float* p3, const Float* p4, const Float* p5,
                   Float* div)
{
  const size_t nc= (size_t) nc_;
  const size_t nczr= 2*(nc/2 + 1);
  for(size_t ix=0; ix<nc; ix++)
    for(size_t iy=0; iy<nc; iy++)
      for(size_t iz=0; iz<nc; iz++) {
        size_t index= (ix*nc + iy)*nczr + iz;
        div[index]=
            p0[index]*(p3[index] + p5[index])
          + p3[index]*p5[index]
          - p1[index]*p1[index]
          - p2[index]*p2[index]
          - p4[index]*p4[index];
      }
}

/* ------------------------------------------------------------------ */
/* Psi(2)(k) from the source, py/lpt.cpp:546-586.                      */
/* ------------------------------------------------------------------ */
void or_lpt_psi2_k(int nc_, double boxsize, const Float* div_k,
                   Float* out0, Float* out1, Float* out2)
{
  const size_t nc= (size_t) nc_;
  const size_t nckz= nc/2 + 1;
  const double dk= 2.0*M_PI/boxsize;
  Float* psi2_k[3]= {out0, out1, out2};

  for(int i=0; i<3; i++) psi2_k[i][0]= psi2_k[i][1]= 0.0;   /* :546-550 */

  for(size_t ix=0; ix<nc; ix++) {
    for(size_t iy=0; iy<nc; iy++) {
      size_t iz0= (ix == 0) && (iy == 0);
      for(size_t iz=iz0; iz<nckz; iz++) {
        size_t index= (ix*nc + iy)*nckz + iz;
        double kvec[3]= {lpt_k(ix, nc, dk), lpt_k(iy, nc, dk),
                         lpt_k(iz, nc, dk)};
        double kmag2= kvec[0]*kvec[0] + kvec[1]*kvec[1] + kvec[2]*kvec[2];
        for(int i=0; i<3; i++) {
          psi2_k[i][2*index    ]=  div_k[2*index + 1]*kvec[i]/kmag2;
          psi2_k[i][2*index + 1]= -div_k[2*index    ]*kvec[i]/kmag2;
        }
      }
    }
  }
}

/* ------------------------------------------------------------------ */
/* Particle grid, lpt_set_displacements py/lpt.cpp:137-211.            */
/* psi*, psi2* are padded real meshes after the inverse transforms     */
/* (still unnormalised: psi2 carries an extra nc^3, :192-193).         */
/* D1, D2, Dv, D2v are Float as at :156-173.                           */
/* ------------------------------------------------------------------ */
void or_lpt_set_particles(int nc_, double boxsize, Float offset,
                          const Float* psi0, const Float* psi1,
                          const Float* psi2_, const Float* q0,
                          const Float* q1, const Float* q2,
                          Float D1, Float D2, Float Dv, Float D2v,
                          Float* x, Float* v, Float* dx1, Float* dx2,
                          uint64_t* id)
{
  const size_t nc= (size_t) nc_;
  const size_t nczr= 2*(nc/2 + 1);
  const Float dx= boxsize/nc;                          /* :144 */
  const double nmesh3_inv= 1.0/pow((double) nc, 3.0); /* :147 */
  const Float* psi[3]= {psi0, psi1, psi2_};
  const Float* psi2[3]= {q0, q1, q2};
  uint64_t pid= 1;
  size_t ip= 0;

  Float xq[3];
  for(size_t ix=0; ix<nc; ix++) {
    xq[0]= (ix + offset)*dx;
    for(size_t iy=0; iy<nc; iy++) {
      xq[1]= (iy + offset)*dx;
      for(size_t iz=0; iz<nc; iz++) {
        xq[2]= (iz + offset)*dx;
        size_t index= (ix*nc + iy)*nczr + iz;
        for(int k=0; k<3; k++) {
          Float dis= psi[k][index];
          Float dis2= nmesh3_inv*psi2[k][index];
          x[3*ip + k]= xq[k] + D1*dis + D2*dis2;
          v[3*ip + k]= Dv*dis + D2v*dis2;
          dx1[3*ip + k]= dis;
          dx2[3*ip + k]= dis2;
        }
        id[ip]= pid++;
        ip++;
      }
    }
  }
}

/* ------------------------------------------------------------------ */
/* cola_velocity, py/cola.cpp:129-148: v + Dv dx1 + D2v dx2 in Float,  */
/* left to right.  The host passes Dv = Dv(a, D1) and                  */
/* D2v = D2v(a, D1): the reference hands D1 to cosmology_D2v_growth    */
/* where D2 is expected (:138), and this keeps that.                   */
/* ------------------------------------------------------------------ */
void or_cola_velocity(const Float* v, const Float* dx1, const Float* dx2,
                      size_t np, Float Dv, Float D2v, Float* out)
{
  for(size_t i=0; i<np; ++i)
    for(size_t k=0; k<3; ++k)
      out[3*i + k]= v[3*i + k] + Dv*dx1[3*i + k] + D2v*dx2[3*i + k];
}

/* ------------------------------------------------------------------ */
/* FP64 variants of the deposit and the gather: the same CIC rule      */
/* (py/pm.cpp:85-115, :156-192) evaluated in double from double        */
/* positions.  They are not the reference's arithmetic; they give the  */
/* FP64 answer that the float32 paths' errors are reported against.    */
/* Serial: a double mesh of n^3 cells is summed in particle order.     */
/* ------------------------------------------------------------------ */
typedef struct {
  size_t i0[3], i1[3];
  double w0[3], w1[3];
} cic64_t;

static inline void cic64_setup(const double* xp, double dx_inv, size_t nc,
                               cic64_t* c)
{
  for(int k=0; k<3; k++) {
    const double X= xp[k]*dx_inv;
    long i0= (long) X;
    const double w1= X - (double) i0;
    if(i0 >= (long) nc) i0= 0;
    if(i0 < 0) i0= 0;
    size_t i1= (size_t) i0 + 1; if(i1 >= nc) i1 -= nc;
    c->i0[k]= (size_t) i0; c->i1[k]= i1;
    c->w0[k]= 1.0 - w1; c->w1[k]= w1;
  }
}

void or_cic_deposit_f64(const double* x, size_t np, double* mesh, int nc_,
                        double boxsize, double pm_factor)
{
  const size_t nc= (size_t) nc_;
  const size_t ncz= 2*(nc/2 + 1);
  const double dx_inv= nc/boxsize;
  const double fac= pm_factor*pm_factor*pm_factor;
  for(size_t ix=0; ix<nc; ix++)
    for(size_t iy=0; iy<nc; iy++)
      for(size_t iz=0; iz<nc; iz++)
        mesh[mesh_index(ix, iy, iz, nc, ncz)]= -1.0;
  for(size_t i=0; i<np; i++) {
    cic64_t c; cic64_setup(x + 3*i, dx_inv, nc, &c);
    for(int o=0; o<8; o++) {
      const int bx= (o >> 2) & 1, by= (o >> 1) & 1, bz= o & 1;
      const size_t jx= bx ? c.i1[0] : c.i0[0];
      const size_t jy= by ? c.i1[1] : c.i0[1];
      const size_t jz= bz ? c.i1[2] : c.i0[2];
      const double w= fac*(bx ? c.w1[0] : c.w0[0])*(by ? c.w1[1] : c.w0[1])*
                      (bz ? c.w1[2] : c.w0[2]);
      mesh[mesh_index(jx, jy, jz, nc, ncz)] += w;
    }
  }
}

void or_force_gather_f64(const double* x, size_t np, const double* fx,
                         int nc_, double boxsize, int axis, double* f,
                         int nthreads)
{
  const size_t nc= (size_t) nc_;
  const size_t ncz= 2*(nc/2 + 1);
  const double dx_inv= nc/boxsize;
  set_threads(nthreads);
#pragma omp parallel for schedule(static) if(nthreads > 1)
  for(size_t i=0; i<np; i++) {
    cic64_t c; cic64_setup(x + 3*i, dx_inv, nc, &c);
    double s= 0.0;
    for(int o=0; o<8; o++) {
      const int bx= (o >> 2) & 1, by= (o >> 1) & 1, bz= o & 1;
      const size_t jx= bx ? c.i1[0] : c.i0[0];
      const size_t jy= by ? c.i1[1] : c.i0[1];
      const size_t jz= bz ? c.i1[2] : c.i0[2];
      s += fx[mesh_index(jx, jy, jz, nc, ncz)]*
           (bx ? c.w1[0] : c.w0[0])*(by ? c.w1[1] : c.w0[1])*
           (bz ? c.w1[2] : c.w0[2]);
    }
    f[3*i + axis]= s;
  }
}

/* Version tag so the harness can detect a stale build. */
int or_version(void) { return 4; }
