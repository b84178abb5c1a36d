/* Stand-in for the adaptive quadrature the reference calls
 * (py/cosmology.cpp:158-168, py/cola.cpp:164-176).  TEST INFRASTRUCTURE
 * (oracle/_ref).  gsl_integration_qag here is an adaptive Gauss-Legendre
 * bisection (oracle/ref_pin/stubs.cpp), converged to about 1e-14 relative
 * whatever tolerance is asked for: the reference's smooth integrands make
 * GSL's own answers that accurate too, so the float-rounded coefficients
 * agree. */
#ifndef FS2REF_GSL_INTEGRATION_H
#define FS2REF_GSL_INTEGRATION_H 1

#include <stddef.h>
#include "gsl_errno.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { double (*function)(double x, void* params); void* params; } gsl_function;
typedef struct fs2ref_workspace { size_t limit; } gsl_integration_workspace;

enum { GSL_INTEG_GAUSS15 = 1, GSL_INTEG_GAUSS21 = 2, GSL_INTEG_GAUSS31 = 3,
       GSL_INTEG_GAUSS41 = 4, GSL_INTEG_GAUSS51 = 5, GSL_INTEG_GAUSS61 = 6 };

gsl_integration_workspace* gsl_integration_workspace_alloc(size_t n);
void gsl_integration_workspace_free(gsl_integration_workspace* w);
int gsl_integration_qag(const gsl_function* f, double a, double b,
                        double epsabs, double epsrel, size_t limit, int key,
                        gsl_integration_workspace* w, double* result,
                        double* abserr);

#ifdef __cplusplus
}
#endif

#endif
