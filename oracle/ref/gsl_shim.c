/* Bodies for the GSL names that the reference's loop.c and config.h refer
 * to. The oracle harness bypasses ray emission (it feeds host-generated rays)
 * and builds no plane sources, so none of these is reached on the compared
 * trace/deposit/solve path; each one stops the process if it ever is. */
#include <stdio.h>
#include <stdlib.h>
#include <gsl/gsl_rng.h>
#include <gsl/gsl_randist.h>

static void unreachable(const char *what) {
	fprintf(stderr, "oracle harness: %s is not part of the compared path\n", what);
	abort();
}
const gsl_rng_type *gsl_rng_mt19937 = NULL;
gsl_rng *gsl_rng_alloc(const gsl_rng_type *T) { (void)T; unreachable("gsl_rng_alloc"); return NULL; }
void gsl_rng_set(const gsl_rng *r, unsigned long int s) { (void)r; (void)s; unreachable("gsl_rng_set"); }
double gsl_rng_uniform(const gsl_rng *r) { (void)r; unreachable("gsl_rng_uniform"); return 0; }
gsl_ran_discrete_t *gsl_ran_discrete_preproc(size_t K, const double *P) { (void)K; (void)P; unreachable("gsl_ran_discrete_preproc"); return NULL; }
size_t gsl_ran_discrete(const gsl_rng *r, const gsl_ran_discrete_t *g) { (void)r; (void)g; unreachable("gsl_ran_discrete"); return 0; }
void gsl_ran_discrete_free(gsl_ran_discrete_t *g) { (void)g; unreachable("gsl_ran_discrete_free"); }
void gsl_ran_dir_3d(const gsl_rng *r, double *x, double *y, double *z) { (void)r; (void)x; (void)y; (void)z; unreachable("gsl_ran_dir_3d"); }
double gsl_ran_flat(const gsl_rng *r, const double a, const double b) { (void)r; (void)a; (void)b; unreachable("gsl_ran_flat"); return 0; }
