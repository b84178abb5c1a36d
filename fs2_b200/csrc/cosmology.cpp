// cosmology.cpp -- host FP64 growth factors of flat LCDM and the COLA drift
// integral.  Follows py/cosmology.cpp:24-171 and py/cola.cpp:152-179 of the
// reference.  The reference integrates with GSL's adaptive Gauss-Kronrod
// (gsl_integration_qag, GK41 at epsrel 5e-9 for D(a), GK61 at epsrel 1e-5 for
// the drift); here an adaptive Gauss-Legendre rule (nodes from Newton's
// iteration on P_n) is driven to a much tighter tolerance, so both agree with
// the true integrals to well below the float rounding the results go through.
#include <cmath>
#include <mutex>
#include <vector>
#include "internal.h"

namespace fs2g {
namespace {

double omega_m0 = 0.0;
double growth_normalisation = 0.0;
constexpr double nLPT = -2.5;   // py/cola.cpp:20

// n-point Gauss-Legendre nodes/weights on [-1,1]
struct GaussLegendre {
  std::vector<double> x, w;
  explicit GaussLegendre(int n) : x(n), w(n) {
    for(int i = 0; i < (n + 1)/2; i++) {
      double z = std::cos(M_PI*(i + 0.75)/(n + 0.5));
      double dp = 0.0;
      for(int it = 0; it < 100; it++) {
        double p0 = 1.0, p1 = z;            // P_0, P_1
        for(int k = 2; k <= n; k++) {
          double p2 = ((2.0*k - 1.0)*z*p1 - (k - 1.0)*p0)/k;
          p0 = p1; p1 = p2;
        }
        dp = n*(z*p1 - p0)/(z*z - 1.0);     // P_n'
        double dz = p1/dp;
        z -= dz;
        if(std::fabs(dz) < 1e-16) break;
      }
      x[i] = -z; x[n - 1 - i] = z;
      w[i] = w[n - 1 - i] = 2.0/((1.0 - z*z)*dp*dp);
    }
  }
  template<class F> double apply(F&& f, double a, double b) const {
    const double c = 0.5*(a + b), h = 0.5*(b - a);
    double s = 0.0;
    for(size_t i = 0; i < x.size(); i++) s += w[i]*f(c + h*x[i]);
    return s*h;
  }
};

const GaussLegendre& gl() {
  static const GaussLegendre rule(20);
  return rule;
}

template<class F>
double adapt(F&& f, double a, double b, double whole, double tol, int depth) {
  const double m = 0.5*(a + b);
  const double left = gl().apply(f, a, m), right = gl().apply(f, m, b);
  const double two = left + right;
  if(depth >= 60 || std::fabs(two - whole) <= tol) return two;
  return adapt(f, a, m, left, 0.5*tol, depth + 1) +
         adapt(f, m, b, right, 0.5*tol, depth + 1);
}

template<class F>
double integrate(F&& f, double a, double b, double epsrel) {
  if(a == b) return 0.0;
  const double whole = gl().apply(f, a, b);
  const double tol = std::fabs(whole)*epsrel + 1e-300;
  return adapt(f, a, b, whole, tol, 0);
}

void check_initialisation() {   // py/cosmology.cpp:134-141
  if(growth_normalisation == 0.0)
    throw Error{FS2G_ERR_RUNTIME, "cosmology module not initialised"};
}

double growth_integrand(double a) {   // py/cosmology.cpp:144-151
  const double aHinv = 1.0/std::sqrt(omega_m0/a + (1 - omega_m0)*(a*a));
  return aHinv*aHinv*aHinv;
}

double growth_unnormalised(double a) {   // py/cosmology.cpp:153-171
  const double r = integrate(growth_integrand, 0.0, a, 1e-14);
  return cosmology_hubble_function(a)*r;
}

}  // namespace

void cosmology_init(double omega_m) {   // py/cosmology.cpp:24-31
  if(!(omega_m > 0.0 && omega_m <= 1.0))
    throw Error{FS2G_ERR_VALUE, "omega_m must be in (0, 1]"};
  omega_m0 = omega_m;
  growth_normalisation = 1.0;             // allow the call below
  growth_normalisation = 1.0/growth_unnormalised(1.0);
}

bool cosmology_initialised() { return growth_normalisation != 0.0; }

double cosmology_omega_m() { check_initialisation(); return omega_m0; }

double cosmology_D_growth(double a) {   // py/cosmology.cpp:33-40
  check_initialisation();
  if(a == 0.0) return 0.0;
  return growth_normalisation*growth_unnormalised(a);
}

double cosmology_D2_growth(double a, double D) {   // :42-48
  if(a == 0.0) return 0.0;
  return -3.0/7.0*D*D*std::pow(cosmology_omega(a), -1.0/143.0);
}

double cosmology_Dv_growth(double a, double D) {   // :50-58
  if(a == 0.0) return 1.0;
  double H = cosmology_hubble_function(a);
  double f = cosmology_f_growth_rate(a);
  return a*a*D*H*f;
}

double cosmology_D2v_growth(double a, double D2) {   // :60-66
  double H = cosmology_hubble_function(a);
  double f = cosmology_f_growth_rate(a);
  return 2.0*a*a*D2*H*f;
}

double cosmology_D2a_growth(double D1, double D2) {   // :68-71
  return D2 - D1*D1;
}

double cosmology_f_growth_rate(double a) {   // :73-84
  check_initialisation();
  if(a == 0.0) return 1.0;
  const double d_un = growth_unnormalised(a);
  const double hf = cosmology_hubble_function(a);
  return 1.0/(d_un*a*a*hf*hf) - 1.5*omega_m0/(hf*hf*a*a*a);
}

double cosmology_hubble_function(double a) {   // :106-110
  return std::sqrt(omega_m0/(a*a*a) + (1 - omega_m0));
}

double cosmology_omega(double a) {   // :112-117
  check_initialisation();
  return omega_m0/(omega_m0 + (1 - omega_m0)*(a*a*a));
}

double cola_Sq(double ai, double af, double av) {   // py/cola.cpp:152-179
  check_initialisation();
  if(!(ai > 0.0))
    throw Error{FS2G_ERR_ASSERTION, "Sq: ai must be positive"};
  const double om = omega_m0;
  auto fun = [om](double a) {
    return std::pow(a, nLPT)/(std::sqrt(om/(a*a*a) + 1.0 - om)*a*a*a);
  };
  const double r = integrate(fun, ai, af, 1e-14);
  return r/std::pow(av, nLPT);
}

// Leapfrog (non-COLA) integrals, py/leapfrog.cpp:97-146: the kick factor
// Sphi = int_ai^af da / (a^2 H(a)) and the drift factor
// Sq = int_ai^af da / (a^3 H(a)), H(a) = sqrt(om/a^3 + 1 - om).
double leapfrog_Sphi(double ai, double af) {
  check_initialisation();
  const double om = omega_m0;
  auto fun = [om](double a) { return 1.0/(std::sqrt(om/(a*a*a) + 1.0 - om)*a*a); };
  return integrate(fun, ai, af, 1e-14);
}

double leapfrog_Sq(double ai, double af) {
  check_initialisation();
  if(!(ai > 0.0))
    throw Error{FS2G_ERR_ASSERTION, "leapfrog drift: a must be positive"};
  const double om = omega_m0;
  auto fun = [om](double a) { return 1.0/(std::sqrt(om/(a*a*a) + 1.0 - om)*a*a*a); };
  return integrate(fun, ai, af, 1e-14);
}

}  // namespace fs2g
