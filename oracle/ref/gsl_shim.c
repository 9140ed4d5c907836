/* Bodies for the GSL names that the reference's loop.c, lte.c, sources.c
 * and config.h refer to. The oracle harness builds no plane sources and
 * draws no uniforms of its own, so the generator calls stop the process if
 * they are ever reached. The discrete distributions are real: lte_fill()
 * (lte.c:46-72) and emit_rays() (loop.c:171-195) build their tables with
 * gsl_ran_discrete_preproc(), and the tests draw from them at chosen
 * uniforms (inverse of the running sum, the same distribution as GSL's
 * Walker tables): one uniform set by oracle_shim_set_uniform(), or a queue
 * of them (oracle_shim_queue_uniforms(), one per draw, in draw order).
 * Directions drawn while emitting source rays (gsl_ran_dir_3d) are not
 * compared and come out as +z. Test infrastructure only. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <gsl/gsl_rng.h>
#include <gsl/gsl_randist.h>
#include <gsl/gsl_eigen.h>

static void unreachable(const char *what) {
	fprintf(stderr, "oracle harness: %s is not part of the compared path\n", what);
	abort();
}
const gsl_rng_type *gsl_rng_mt19937 = NULL;
gsl_rng *gsl_rng_alloc(const gsl_rng_type *T) { (void)T; unreachable("gsl_rng_alloc"); return NULL; }
void gsl_rng_set(const gsl_rng *r, unsigned long int s) { (void)r; (void)s; unreachable("gsl_rng_set"); }
double gsl_rng_uniform(const gsl_rng *r) { (void)r; unreachable("gsl_rng_uniform"); return 0; }
static double shim_uniform = 0.0;
static const double *shim_queue = NULL;
static size_t shim_queue_n = 0, shim_queue_pos = 0;
void oracle_shim_set_uniform(double u) { shim_uniform = u; }
void oracle_shim_queue_uniforms(const double *u, size_t n) {
	shim_queue = u;
	shim_queue_n = n;
	shim_queue_pos = 0;
}
static double next_uniform(void) {
	if (!shim_queue) return shim_uniform;
	if (shim_queue_pos >= shim_queue_n) unreachable("a draw past the queued uniforms");
	return shim_queue[shim_queue_pos++];
}
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
	const double target = next_uniform() * total;
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
void gsl_ran_dir_3d(const gsl_rng *r, double *x, double *y, double *z) {
	(void)r;
	if (!shim_queue) unreachable("gsl_ran_dir_3d");
	*x = 0.0;
	*y = 0.0;
	*z = 1.0;
}
double gsl_ran_flat(const gsl_rng *r, const double a, const double b) { (void)r; (void)a; (void)b; unreachable("gsl_ran_flat"); return 0; }

/* gsl_eigen.h stand-ins (plane sources only; never reached) */
gsl_matrix_view gsl_matrix_view_array(double *base, size_t n1, size_t n2) {
	(void)base; (void)n1; (void)n2; unreachable("gsl_matrix_view_array"); gsl_matrix_view v = {{0, 0, 0}}; return v;
}
gsl_vector *gsl_vector_alloc(size_t n) { (void)n; unreachable("gsl_vector_alloc"); return NULL; }
gsl_matrix *gsl_matrix_alloc(size_t n1, size_t n2) { (void)n1; (void)n2; unreachable("gsl_matrix_alloc"); return NULL; }
gsl_eigen_symmv_workspace *gsl_eigen_symmv_alloc(size_t n) { (void)n; unreachable("gsl_eigen_symmv_alloc"); return NULL; }
int gsl_eigen_symmv(gsl_matrix *A, gsl_vector *e, gsl_matrix *v, gsl_eigen_symmv_workspace *w) {
	(void)A; (void)e; (void)v; (void)w; unreachable("gsl_eigen_symmv"); return 0;
}
int gsl_eigen_symmv_sort(gsl_vector *e, gsl_matrix *v, int t) { (void)e; (void)v; (void)t; unreachable("gsl_eigen_symmv_sort"); return 0; }
gsl_vector_view gsl_matrix_column(gsl_matrix *m, size_t j) {
	(void)m; (void)j; unreachable("gsl_matrix_column"); gsl_vector_view v = {{0, 0}}; return v;
}
double gsl_vector_get(const gsl_vector *v, size_t i) { (void)v; (void)i; unreachable("gsl_vector_get"); return 0; }
void gsl_matrix_free(gsl_matrix *m) { (void)m; }
void gsl_vector_free(gsl_vector *v) { (void)v; }
void gsl_eigen_symmv_free(gsl_eigen_symmv_workspace *w) { (void)w; }
