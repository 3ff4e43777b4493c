#ifndef GG_SHIM_GSL_RNG_H
#define GG_SHIM_GSL_RNG_H
#include <stddef.h>
/* splitmix64 stream in place of GSL's ranlxd1 (not bit-identical to GSL) */
typedef struct { int id; } gsl_rng_type;
typedef struct { unsigned long long state; } gsl_rng;
extern const gsl_rng_type *gsl_rng_ranlxd1;
gsl_rng *gsl_rng_alloc(const gsl_rng_type *t);
void gsl_rng_free(gsl_rng *r);
void gsl_rng_set(gsl_rng *r, unsigned long seed);
double gsl_rng_uniform(gsl_rng *r);
size_t gsl_rng_size(const gsl_rng *r);
void *gsl_rng_state(const gsl_rng *r);
#endif
