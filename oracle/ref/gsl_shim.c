/* Bodies for the GSL names that the reference's loop.c, lte.c and config.h
 * refer to. The oracle harness bypasses ray emission (it feeds
 * host-generated rays) and builds no plane sources, so the generator calls
 * stop the process if they are ever reached. The discrete distributions
 * are real: lte_fill() (lte.c:46-72) builds its tables with
 * gsl_ran_discrete_preproc(), and the tests read their weights back and
 * draw from them at chosen uniforms (inverse of the running sum, the same
 * distribution as GSL's Walker tables). Test infrastructure only. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
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
static double shim_uniform = 0.0;
void oracle_shim_set_uniform(double u) { shim_uniform = u; }
gsl_ran_discrete_t *gsl_ran_discrete_preproc(size_t K, const double *P) {
	gsl_ran_discrete_t *g = malloc(sizeof *g);
	g->K = K;
	g->P = malloc(sizeof(double) * K);
	memcpy(g->P, P, sizeof(double) * K);
	return g;
}
size_t gsl_ran_discrete(const gsl_rng *r, const gsl_ran_discrete_t *g) {
	(void)r;
	double total = 0.0;
	for (size_t i = 0; i < g->K; i++) total += g->P[i];
	const double target = shim_uniform * total;
	double acc = 0.0;
	size_t last = 0;
	for (size_t i = 0; i < g->K; i++) {
		acc += g->P[i];
		if (g->P[i] > 0.0) last = i;
		if (acc > target) return i;
	}
	return last;
}
void gsl_ran_discrete_free(gsl_ran_discrete_t *g) {
	if (!g) return;
	free(g->P);
	free(g);
}
void gsl_ran_dir_3d(const gsl_rng *r, double *x, double *y, double *z) { (void)r; (void)x; (void)y; (void)z; unreachable("gsl_ran_dir_3d"); }
double gsl_ran_flat(const gsl_rng *r, const double a, const double b) { (void)r; (void)a; (void)b; unreachable("gsl_ran_flat"); return 0; }
