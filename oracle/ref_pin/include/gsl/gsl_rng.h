/* Stand-in for <gsl/gsl_rng.h>.  TEST INFRASTRUCTURE (oracle/_ref).
 *
 * NOT GSL's ranlxd1: gsl_rng_uniform returns a SplitMix64 stream keyed by
 * the value given to gsl_rng_set (oracle/ref_pin/stubs.cpp).  What matters
 * for the pin is that every draw the reference makes is recorded in order
 * (with the seed it was made under), so the oracle can be fed exactly the
 * draws the reference used. */
#ifndef FS2REF_GSL_RNG_H
#define FS2REF_GSL_RNG_H 1

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fs2ref_rng_type { const char* name; } gsl_rng_type;
typedef struct fs2ref_rng { unsigned long long state; unsigned long seed; } gsl_rng;

extern const gsl_rng_type* gsl_rng_ranlxd1;

gsl_rng* gsl_rng_alloc(const gsl_rng_type* t);
void gsl_rng_set(gsl_rng* r, unsigned long seed);
double gsl_rng_uniform(gsl_rng* r);
void gsl_rng_free(gsl_rng* r);

#ifdef __cplusplus
}
#endif

#endif
