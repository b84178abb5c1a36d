/* Stand-in for the natural cubic spline the reference's PowerSpectrum uses
 * (py/power.cpp:31-55).  TEST INFRASTRUCTURE (oracle/_ref).  The spline is
 * the standard natural cubic spline (second derivatives zero at both ends,
 * tridiagonal solve), oracle/ref_pin/stubs.cpp. */
#ifndef FS2REF_GSL_SPLINE_H
#define FS2REF_GSL_SPLINE_H 1

#include <stddef.h>
#include "gsl_errno.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fs2ref_interp_type { const char* name; unsigned min_size; } gsl_interp_type;
typedef struct fs2ref_interp { size_t n; double* m; } gsl_interp;
typedef struct fs2ref_accel { size_t cache; } gsl_interp_accel;

extern const gsl_interp_type* gsl_interp_cspline;

gsl_interp* gsl_interp_alloc(const gsl_interp_type* t, size_t n);
unsigned int gsl_interp_min_size(const gsl_interp* interp);
int gsl_interp_init(gsl_interp* interp, const double xa[], const double ya[],
                    size_t n);
double gsl_interp_eval(const gsl_interp* interp, const double xa[],
                       const double ya[], double x, gsl_interp_accel* a);
void gsl_interp_free(gsl_interp* interp);
gsl_interp_accel* gsl_interp_accel_alloc(void);
void gsl_interp_accel_free(gsl_interp_accel* a);

#ifdef __cplusplus
}
#endif

#endif
