/* Stand-in for <gsl/gsl_errno.h>.  TEST INFRASTRUCTURE (oracle/_ref). */
#ifndef FS2REF_GSL_ERRNO_H
#define FS2REF_GSL_ERRNO_H 1
#define GSL_SUCCESS 0
#define GSL_EDOM 1
#endif
