// power.cpp -- linear power spectrum table, follows py/power.cpp:15-170.
// The table is read as the reference reads it; ln P(ln k) is interpolated by
// a natural cubic spline (the reference uses gsl_interp_cspline, whose end
// conditions are natural too), solved here by the tridiagonal (Thomas)
// algorithm.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include "internal.h"

using fs2g::Error;

double fs2g_power::eval_logP(double lk) const {
  int lo = 0, hi = n - 1;
  if(lk <= log_k[0]) lo = 0;
  else if(lk >= log_k[hi]) lo = hi - 1;
  else {
    while(hi - lo > 1) {
      int mid = (lo + hi)/2;
      if(log_k[mid] > lk) hi = mid; else lo = mid;
    }
  }
  const double t = lk - log_k[lo];
  return sa[lo] + t*(sb[lo] + t*(sc[lo] + t*sd[lo]));
}

namespace fs2g {

void power_build_spline(fs2g_power* ps) {
  const int n = ps->n;
  if(n < 3)   // gsl_interp_min_size for cspline (py/power.cpp:34-36)
    throw Error{FS2G_ERR_IO, "not enough power spectrum data points for a "
                             "cubic spline (need 3)"};
  const std::vector<double>& x = ps->log_k;
  const std::vector<double>& y = ps->log_P;
  // second derivatives M with M[0] = M[n-1] = 0
  std::vector<double> M(n, 0.0), cp(n, 0.0), dp(n, 0.0);
  for(int i = 1; i < n - 1; i++) {
    const double h0 = x[i] - x[i-1], h1 = x[i+1] - x[i];
    const double a = h0, b = 2.0*(h0 + h1), c = h1;
    const double r = 6.0*((y[i+1] - y[i])/h1 - (y[i] - y[i-1])/h0);
    const double denom = b - a*cp[i-1];
    cp[i] = c/denom;
    dp[i] = (r - a*dp[i-1])/denom;
  }
  for(int i = n - 2; i >= 1; i--) M[i] = dp[i] - cp[i]*M[i+1];
  ps->sa.assign(n - 1, 0.0); ps->sb.assign(n - 1, 0.0);
  ps->sc.assign(n - 1, 0.0); ps->sd.assign(n - 1, 0.0);
  for(int i = 0; i < n - 1; i++) {
    const double h = x[i+1] - x[i];
    ps->sa[i] = y[i];
    ps->sb[i] = (y[i+1] - y[i])/h - h*(2.0*M[i] + M[i+1])/6.0;
    ps->sc[i] = 0.5*M[i];
    ps->sd[i] = (M[i+1] - M[i])/(6.0*h);
  }
}

}  // namespace fs2g

// ---------------------------------------------------------------------
// ABI
// ---------------------------------------------------------------------
extern "C" {

int fs2g_power_alloc(const char* filename, fs2g_power** out) {
  // PowerSpectrum::read_file_, py/power.cpp:57-144
  if(!filename || !out) return fs2g::fail(FS2G_ERR_VALUE, "null argument");
  FILE* fp = std::fopen(filename, "r");
  if(!fp)
    return fs2g::fail(FS2G_ERR_IO, std::string("unable to open input power "
                                               "spectrum file: ") + filename);
  std::vector<double> ks, Ps;
  char line[128];
  double k_prev = 0.0;
  while(std::fgets(line, 127, fp)) {
    if(line[0] == '#') continue;
    double k, P;
    if(std::sscanf(line, "%lg %lg", &k, &P) != 2) break;   // :98-104
    if(k <= 0.0) continue;                                 // :106-109
    if(k < k_prev) {                                       // :111-117
      std::fclose(fp);
      return fs2g::fail(FS2G_ERR_IO, "wavenumber k in the power spectrum "
                                     "file must be sorted in increasing order");
    }
    ks.push_back(k); Ps.push_back(P);
    k_prev = k;
  }
  std::fclose(fp);
  return fs2g_power_from_table(ks.data(), Ps.data(), (int) ks.size(), out);
}

int fs2g_power_from_table(const double* k, const double* P, int n,
                          fs2g_power** out) {
  if(!out || (n > 0 && (!k || !P)))
    return fs2g::fail(FS2G_ERR_VALUE, "null argument");
  try {
    fs2g_power* ps = new fs2g_power();
    ps->n = n;
    ps->log_k.resize(n); ps->log_P.resize(n);
    for(int j = 0; j < n; j++) {                          // :135-138
      if(!(k[j] > 0.0) || !(P[j] > 0.0) || (j > 0 && !(k[j] > k[j-1]))) {
        delete ps;
        return fs2g::fail(FS2G_ERR_IO, "power spectrum table needs k > 0 "
                          "strictly increasing and P > 0");
      }
      ps->log_k[j] = std::log(k[j]);
      ps->log_P[j] = std::log(P[j]);
    }
    try { fs2g::power_build_spline(ps); }
    catch(...) { delete ps; throw; }
    *out = ps;
    return FS2G_OK;
  }
  catch(const fs2g::Error& e) { return fs2g::fail(e.code, e.msg); }
  catch(const std::bad_alloc&) { return fs2g::fail(FS2G_ERR_MEMORY, "out of host memory"); }
}

int fs2g_power_free(fs2g_power* ps) { delete ps; return FS2G_OK; }

int fs2g_power_n(const fs2g_power* ps, int* n) {
  if(!ps || !n) return fs2g::fail(FS2G_ERR_VALUE, "null argument");
  *n = ps->n;
  return FS2G_OK;
}

int fs2g_power_i(const fs2g_power* ps, int i, double* k, double* P) {
  if(!ps) return fs2g::fail(FS2G_ERR_VALUE, "null argument");
  if(i < 0 || i >= ps->n) return fs2g::fail(FS2G_ERR_INDEX, "index out of range");
  if(k) *k = std::exp(ps->log_k[i]);
  if(P) *P = std::exp(ps->log_P[i]);
  return FS2G_OK;
}

int fs2g_power_P(const fs2g_power* ps, double k, double* P) {
  // PowerSpectrum::P, py/power.cpp:50-55; outside the table GSL reports a
  // domain error, and so does this
  if(!ps || !P) return fs2g::fail(FS2G_ERR_VALUE, "null argument");
  const double lk = std::log(k);
  if(!(lk >= ps->log_k.front() && lk <= ps->log_k.back()))
    return fs2g::fail(FS2G_ERR_VALUE, "k outside the power spectrum table");
  *P = std::exp(ps->eval_logP(lk));
  return FS2G_OK;
}

int fs2g_power_sigma(const fs2g_power* ps, double R, double* sigma) {
  // PowerSpectrum::compute_sigma, py/power.cpp:146-170
  if(!ps || !sigma) return fs2g::fail(FS2G_ERR_VALUE, "null argument");
  const double fac = 1.0/(2.0*M_PI*M_PI);
  double k0 = std::exp(ps->log_k[0]);
  double f0 = 0.0, sigma2 = 0.0;
  for(int i = 0; i < ps->n; i++) {
    double k = std::exp(ps->log_k[i]);
    double x = k*R;
    double w = 3.0*(std::sin(x) - x*std::cos(x))/(x*x*x);
    double f1 = std::exp(ps->log_P[i])*k*k*w*w;
    sigma2 += 0.5*(f0 + f1)*(k - k0);
    k0 = k;
    f0 = f1;
  }
  *sigma = std::sqrt(fac*sigma2);
  return FS2G_OK;
}

}  // extern "C"
