/* Minimal stand-in for the GSL random-number header, written for the oracle
 * harness. The reference includes <gsl/gsl_rng.h> from config.h and loop.c;
 * only the type names and prototypes are needed to compile those files. The
 * harness feeds host-generated rays, so none of these functions is called on
 * the compared trace/deposit/solve path (ray emission is bypassed). */
#ifndef ORACLE_GSL_RNG_H
#define ORACLE_GSL_RNG_H
typedef struct gsl_rng_type gsl_rng_type;
typedef struct gsl_rng gsl_rng;
extern const gsl_rng_type *gsl_rng_mt19937;
gsl_rng *gsl_rng_alloc(const gsl_rng_type *T);
void gsl_rng_set(const gsl_rng *r, unsigned long int seed);
double gsl_rng_uniform(const gsl_rng *r);
#endif
