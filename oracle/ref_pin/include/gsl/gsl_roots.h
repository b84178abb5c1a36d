/* Empty stand-in: included by the reference's sources, nothing from it is
 * called on the PM / COLA / 2LPT path.  TEST INFRASTRUCTURE (oracle/_ref). */
#ifndef FS2REF_GSL_ROOTS_H
#define FS2REF_GSL_ROOTS_H 1
#include "gsl_errno.h"
#endif
