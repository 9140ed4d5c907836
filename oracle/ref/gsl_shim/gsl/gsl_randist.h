/* Minimal stand-in for GSL's distribution header (prototypes only); see
 * gsl_rng.h in this directory for why nothing here is on the compared path. */
#ifndef ORACLE_GSL_RANDIST_H
#define ORACLE_GSL_RANDIST_H
#include <stddef.h>
#include <gsl/gsl_rng.h>
/* A discrete distribution keeps its weights; a draw inverts their running
 * sum at the uniform set by oracle_shim_set_uniform() (gsl_shim.c). */
typedef struct gsl_ran_discrete_t {
	size_t K;
	double *P;
} gsl_ran_discrete_t;
void oracle_shim_set_uniform(double u);
void oracle_shim_queue_uniforms(const double *u, size_t n);
gsl_ran_discrete_t *gsl_ran_discrete_preproc(size_t K, const double *P);
size_t gsl_ran_discrete(const gsl_rng *r, const gsl_ran_discrete_t *g);
void gsl_ran_discrete_free(gsl_ran_discrete_t *g);
void gsl_ran_dir_3d(const gsl_rng *r, double *x, double *y, double *z);
double gsl_ran_flat(const gsl_rng *r, const double a, const double b);
#endif
