// stubs.cpp -- single-rank stand-ins for the third-party calls of the
// reference's PM / COLA / 2LPT sources (FFTW 3 MPI, GSL rng / quadrature /
// cubic spline).  TEST INFRASTRUCTURE: linked only into oracle/_ref, the
// build of the reference's own loops that pins the oracle.  Nothing here is
// FFTW's or GSL's code; each routine is written from the mathematics:
//
//  * 3-D real DFTs as separable 1-D DFTs in double (radix-2 for powers of
//    two, the direct sum otherwise), rounded to float on output;
//  * adaptive Gauss-Legendre quadrature with nodes from Newton's iteration
//    on the Legendre polynomial;
//  * the natural cubic spline (tridiagonal solve for the second
//    derivatives);
//  * SplitMix64 (Steele, Lea, Flood 2014) as the uniform stream, with a log
//    of every draw.
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "fftw3-mpi.h"
#include "gsl/gsl_integration.h"
#include "gsl/gsl_rng.h"
#include "gsl/gsl_spline.h"

typedef std::complex<double> cd;

// ------------------------------------------------------------------ FFT
struct fs2ref_plan {
  ptrdiff_t n0, n1, n2;
  int inverse;          // 0: r2c, 1: c2r
  int transposed;       // spectrum stored [n1][n0][n2/2+1]
};

// hooks a harness may install: `before` runs first and, when it returns
// nonzero, the built-in transform is skipped; `after` runs last.  Both get
// the plan's shape and the real / complex arrays.
typedef int (*fs2ref_fft_hook)(void* ctx, int inverse, int n0, int n1, int n2,
                               int transposed, float* real, float* cplx);
static fs2ref_fft_hook g_before = nullptr, g_after = nullptr;
static void* g_hook_ctx = nullptr;

extern "C" void fs2ref_set_fft_hooks(fs2ref_fft_hook before,
                                     fs2ref_fft_hook after, void* ctx) {
  g_before = before; g_after = after; g_hook_ctx = ctx;
}

// in-place 1-D DFT of length n with stride 1 (sign -1 forward, +1 inverse)
static void dft1(cd* a, size_t n, int sign, std::vector<cd>& tmp) {
  if(n <= 1) return;
  if((n & (n - 1)) == 0) {
    // iterative radix-2, bit-reversed input order
    for(size_t i = 1, j = 0; i < n; i++) {
      size_t bit = n >> 1;
      for(; j & bit; bit >>= 1) j ^= bit;
      j ^= bit;
      if(i < j) std::swap(a[i], a[j]);
    }
    for(size_t len = 2; len <= n; len <<= 1) {
      const double ang = sign*2.0*M_PI/(double) len;
      for(size_t i = 0; i < n; i += len)
        for(size_t k = 0; k < len/2; k++) {
          const cd w(std::cos(ang*(double) k), std::sin(ang*(double) k));
          const cd u = a[i + k], v = a[i + k + len/2]*w;
          a[i + k] = u + v;
          a[i + k + len/2] = u - v;
        }
    }
    return;
  }
  tmp.assign(n, cd(0.0, 0.0));
  for(size_t k = 0; k < n; k++) {
    cd s(0.0, 0.0);
    for(size_t j = 0; j < n; j++) {
      const double ang = sign*2.0*M_PI*(double)((j*k) % n)/(double) n;
      s += a[j]*cd(std::cos(ang), std::sin(ang));
    }
    tmp[k] = s;
  }
  std::copy(tmp.begin(), tmp.end(), a);
}

// transform axis `ax` (0: x, 1: y, 2: z) of a [N0][N1][N2] complex array
static void dft_axis(std::vector<cd>& A, size_t N0, size_t N1, size_t N2,
                     int ax, int sign) {
  const size_t len = ax == 0 ? N0 : (ax == 1 ? N1 : N2);
  const size_t stride = ax == 0 ? N1*N2 : (ax == 1 ? N2 : 1);
  std::vector<cd> line(len), tmp;
  for(size_t i = 0; i < N0; i++)
    for(size_t j = 0; j < N1; j++)
      for(size_t k = 0; k < N2; k++) {
        const size_t c[3] = {i, j, k};
        if(c[ax] != 0) continue;
        const size_t base = (i*N1 + j)*N2 + k;
        for(size_t m = 0; m < len; m++) line[m] = A[base + m*stride];
        dft1(line.data(), len, sign, tmp);
        for(size_t m = 0; m < len; m++) A[base + m*stride] = line[m];
      }
}

static size_t spec_index(const fs2ref_plan* p, size_t kx, size_t ky,
                         size_t kz) {
  const size_t nk = (size_t) p->n2/2 + 1;
  return p->transposed ? ((ky*(size_t) p->n0 + kx)*nk + kz)
                       : ((kx*(size_t) p->n1 + ky)*nk + kz);
}

static void exec_r2c(const fs2ref_plan* p, const float* in, float* out) {
  const size_t n0 = p->n0, n1 = p->n1, n2 = p->n2, nk = n2/2 + 1;
  const size_t ncz = 2*nk;
  std::vector<cd> A(n0*n1*n2);
  for(size_t i = 0; i < n0; i++)
    for(size_t j = 0; j < n1; j++)
      for(size_t k = 0; k < n2; k++)
        A[(i*n1 + j)*n2 + k] = cd((double) in[(i*n1 + j)*ncz + k], 0.0);
  for(int ax = 2; ax >= 0; ax--) dft_axis(A, n0, n1, n2, ax, -1);
  for(size_t i = 0; i < n0; i++)
    for(size_t j = 0; j < n1; j++)
      for(size_t k = 0; k < nk; k++) {
        const cd v = A[(i*n1 + j)*n2 + k];
        const size_t o = spec_index(p, i, j, k);
        out[2*o] = (float) v.real();
        out[2*o + 1] = (float) v.imag();
      }
}

static void exec_c2r(const fs2ref_plan* p, const float* in, float* out) {
  const size_t n0 = p->n0, n1 = p->n1, n2 = p->n2, nk = n2/2 + 1;
  const size_t ncz = 2*nk;
  std::vector<cd> B(n0*n1*nk);
  for(size_t i = 0; i < n0; i++)
    for(size_t j = 0; j < n1; j++)
      for(size_t k = 0; k < nk; k++) {
        const size_t o = spec_index(p, i, j, k);
        B[(i*n1 + j)*nk + k] = cd((double) in[2*o], (double) in[2*o + 1]);
      }
  dft_axis(B, n0, n1, nk, 0, +1);
  dft_axis(B, n0, n1, nk, 1, +1);
  // along z: real part of the Hermitian extension (imaginary parts of the
  // kz = 0 and kz = n2/2 bins do not enter)
  std::vector<double> r(n2);
  for(size_t i = 0; i < n0; i++)
    for(size_t j = 0; j < n1; j++) {
      const cd* row = &B[(i*n1 + j)*nk];
      for(size_t z = 0; z < n2; z++) {
        double s = row[0].real();
        for(size_t k = 1; k < nk; k++) {
          const double ang = 2.0*M_PI*(double)((k*z) % n2)/(double) n2;
          const double re = row[k].real()*std::cos(ang) -
                            row[k].imag()*std::sin(ang);
          s += (2*k == n2) ? re : 2.0*re;
        }
        r[z] = s;
      }
      float* o = out + (i*n1 + j)*ncz;
      for(size_t z = 0; z < n2; z++) o[z] = (float) r[z];
      for(size_t z = n2; z < ncz; z++) o[z] = 0.0f;
    }
}

extern "C" {

ptrdiff_t fftwf_mpi_local_size_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2,
                                  MPI_Comm, ptrdiff_t* local_n0,
                                  ptrdiff_t* local_0_start) {
  *local_n0 = n0; *local_0_start = 0;
  return n0*n1*n2;                       // n2 is already n/2 + 1 here
}

ptrdiff_t fftwf_mpi_local_size_3d_transposed(
    ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, MPI_Comm, ptrdiff_t* local_n0,
    ptrdiff_t* local_0_start, ptrdiff_t* local_n1, ptrdiff_t* local_1_start) {
  *local_n0 = n0; *local_0_start = 0;
  *local_n1 = n1; *local_1_start = 0;
  return n0*n1*n2;
}

fftwf_plan fftwf_mpi_plan_dft_r2c_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2,
                                     float*, fftwf_complex*, MPI_Comm,
                                     unsigned flags) {
  fs2ref_plan* p = new fs2ref_plan{n0, n1, n2, 0,
                                   (flags & FFTW_MPI_TRANSPOSED_OUT) ? 1 : 0};
  return p;
}

fftwf_plan fftwf_mpi_plan_dft_c2r_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2,
                                     fftwf_complex*, float*, MPI_Comm,
                                     unsigned flags) {
  fs2ref_plan* p = new fs2ref_plan{n0, n1, n2, 1,
                                   (flags & FFTW_MPI_TRANSPOSED_IN) ? 1 : 0};
  return p;
}

void fftwf_mpi_execute_dft_r2c(fftwf_plan p, float* in, fftwf_complex* out) {
  float* o = reinterpret_cast<float*>(out);
  if(g_before && g_before(g_hook_ctx, 0, (int) p->n0, (int) p->n1,
                          (int) p->n2, p->transposed, in, o))
    ;
  else {
    // in place (in == out) in the reference: read everything first
    const size_t ncz = 2*((size_t) p->n2/2 + 1);
    std::vector<float> copy(in, in + (size_t) p->n0*p->n1*ncz);
    exec_r2c(p, copy.data(), o);
  }
  if(g_after) g_after(g_hook_ctx, 0, (int) p->n0, (int) p->n1, (int) p->n2,
                      p->transposed, in, o);
}

void fftwf_mpi_execute_dft_c2r(fftwf_plan p, fftwf_complex* in, float* out) {
  float* c = reinterpret_cast<float*>(in);
  if(g_before && g_before(g_hook_ctx, 1, (int) p->n0, (int) p->n1,
                          (int) p->n2, p->transposed, out, c))
    ;
  else {
    const size_t nk = (size_t) p->n2/2 + 1;
    std::vector<float> copy(c, c + 2*(size_t) p->n0*p->n1*nk);
    exec_c2r(p, copy.data(), out);
  }
  if(g_after) g_after(g_hook_ctx, 1, (int) p->n0, (int) p->n1, (int) p->n2,
                      p->transposed, out, c);
}

void fftwf_destroy_plan(fftwf_plan p) { delete p; }
void fftwf_mpi_init(void) {}
void fftwf_mpi_cleanup(void) {}
void* fftwf_malloc(size_t n) { return std::malloc(n ? n : 1); }
void fftwf_free(void* p) { std::free(p); }

// ------------------------------------------------------------------ rng
static const gsl_rng_type ranlxd1_standin = {"splitmix64 stand-in"};
const gsl_rng_type* gsl_rng_ranlxd1 = &ranlxd1_standin;

struct DrawLog { std::vector<unsigned long> seed; std::vector<double> u; };
static DrawLog g_draws;

void fs2ref_rng_log_clear(void) { g_draws.seed.clear(); g_draws.u.clear(); }
size_t fs2ref_rng_log_size(void) { return g_draws.u.size(); }
void fs2ref_rng_log_copy(unsigned long* seeds, double* u) {
  std::memcpy(seeds, g_draws.seed.data(), g_draws.seed.size()*sizeof(unsigned long));
  std::memcpy(u, g_draws.u.data(), g_draws.u.size()*sizeof(double));
}

gsl_rng* gsl_rng_alloc(const gsl_rng_type*) {
  gsl_rng* r = new gsl_rng;
  r->state = 0; r->seed = 0;
  return r;
}
void gsl_rng_set(gsl_rng* r, unsigned long seed) { r->state = seed; r->seed = seed; }
double gsl_rng_uniform(gsl_rng* r) {
  uint64_t z = (r->state += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30))*0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27))*0x94D049BB133111EBull;
  z ^= z >> 31;
  const double u = (double)(z >> 11)*(1.0/9007199254740992.0);   // [0, 1)
  g_draws.seed.push_back(r->seed);
  g_draws.u.push_back(u);
  return u;
}
void gsl_rng_free(gsl_rng* r) { delete r; }

// ------------------------------------------------------------------ quadrature
static const int GL_N = 20;
static double gl_x[GL_N], gl_w[GL_N];
static bool gl_ready = false;

static void gl_init() {
  // nodes of P_20 by Newton's iteration from Chebyshev guesses
  for(int i = 0; i < GL_N; i++) {
    double x = std::cos(M_PI*(i + 0.75)/(GL_N + 0.5)), dp = 0.0;
    for(int it = 0; it < 100; it++) {
      double p0 = 1.0, p1 = x;
      for(int k = 2; k <= GL_N; k++) {
        const double p2 = ((2*k - 1)*x*p1 - (k - 1)*p0)/k;
        p0 = p1; p1 = p2;
      }
      dp = GL_N*(x*p1 - p0)/(x*x - 1.0);
      const double dx = p1/dp;
      x -= dx;
      if(std::fabs(dx) < 1e-16) break;
    }
    gl_x[i] = x;
    gl_w[i] = 2.0/((1.0 - x*x)*dp*dp);
  }
  gl_ready = true;
}

static double gl_rule(const gsl_function* f, double a, double b) {
  const double c = 0.5*(a + b), h = 0.5*(b - a);
  double s = 0.0;
  for(int i = 0; i < GL_N; i++) s += gl_w[i]*f->function(c + h*gl_x[i], f->params);
  return s*h;
}

static double gl_adapt(const gsl_function* f, double a, double b, double whole,
                       int depth) {
  const double m = 0.5*(a + b);
  const double l = gl_rule(f, a, m), r = gl_rule(f, m, b);
  if(depth >= 48 || std::fabs(l + r - whole) <= 1e-15*std::fabs(l + r) + 1e-300)
    return l + r;
  return gl_adapt(f, a, m, l, depth + 1) + gl_adapt(f, m, b, r, depth + 1);
}

gsl_integration_workspace* gsl_integration_workspace_alloc(size_t n) {
  return new gsl_integration_workspace{n};
}
void gsl_integration_workspace_free(gsl_integration_workspace* w) { delete w; }

int gsl_integration_qag(const gsl_function* f, double a, double b, double,
                        double, size_t, int, gsl_integration_workspace*,
                        double* result, double* abserr) {
  if(!gl_ready) gl_init();
  *result = gl_adapt(f, a, b, gl_rule(f, a, b), 0);
  *abserr = 0.0;
  return GSL_SUCCESS;
}

// ------------------------------------------------------------------ spline
static const gsl_interp_type cspline_type = {"natural cubic spline", 3};
const gsl_interp_type* gsl_interp_cspline = &cspline_type;

gsl_interp* gsl_interp_alloc(const gsl_interp_type*, size_t n) {
  gsl_interp* s = new gsl_interp;
  s->n = n;
  s->m = new double[n];
  return s;
}
unsigned int gsl_interp_min_size(const gsl_interp*) { return 3; }

int gsl_interp_init(gsl_interp* s, const double x[], const double y[],
                    size_t n) {
  // second derivatives m: natural ends, Thomas algorithm
  std::vector<double> c(n, 0.0), d(n, 0.0);
  s->m[0] = s->m[n - 1] = 0.0;
  for(size_t i = 1; i + 1 < n; i++) {
    const double h0 = x[i] - x[i - 1], h1 = x[i + 1] - x[i];
    const double a = h0, b = 2.0*(h0 + h1), cc = h1;
    const double r = 6.0*((y[i + 1] - y[i])/h1 - (y[i] - y[i - 1])/h0);
    const double den = b - a*c[i - 1];
    c[i] = cc/den;
    d[i] = (r - a*d[i - 1])/den;
  }
  for(size_t i = n - 2; i >= 1; i--) {
    s->m[i] = d[i] - c[i]*s->m[i + 1];
    if(i == 1) break;
  }
  return GSL_SUCCESS;
}

double gsl_interp_eval(const gsl_interp* s, const double x[], const double y[],
                       double xi, gsl_interp_accel*) {
  const size_t n = s->n;
  if(!(xi >= x[0] && xi <= x[n - 1])) return std::nan("");
  size_t lo = 0, hi = n - 1;
  while(hi - lo > 1) {
    const size_t mid = (lo + hi)/2;
    if(x[mid] > xi) hi = mid; else lo = mid;
  }
  const double h = x[hi] - x[lo];
  const double A = (x[hi] - xi)/h, B = (xi - x[lo])/h;
  return A*y[lo] + B*y[hi] +
         ((A*A*A - A)*s->m[lo] + (B*B*B - B)*s->m[hi])*h*h/6.0;
}

void gsl_interp_free(gsl_interp* s) { delete[] s->m; delete s; }
gsl_interp_accel* gsl_interp_accel_alloc(void) { return new gsl_interp_accel{0}; }
void gsl_interp_accel_free(gsl_interp_accel* a) { delete a; }

}  // extern "C"
