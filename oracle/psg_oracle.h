/* CPU restatement of psphray's trace -> deposit -> merge -> update hot path.
 *
 * TEST INFRASTRUCTURE ONLY: this is the checker the CUDA path is compared
 * against. Only tests, the smoke check and the CPU-baseline leg of the bench
 * may load it; the product never links it.
 *
 * Parity is pinned against the reference itself: the same cases run through
 * oracle/_ref/libpsphray_ref.so (the reference's own sources) in the tests. */
#ifndef PSG_ORACLE_H
#define PSG_ORACLE_H
#include <stddef.h>
#include <stdint.h>

typedef struct {
	float s[3];
	float dir[3];
	double Nph;
	double freq;
	double length;
} po_ray;

typedef struct {
	int64_t ipar;
	double d;
	double b;
} po_hit;

/* Tables after unit scaling, as the reference holds them (tabfun.h TabFun).
 * Rate columns, in this order: HIci HIIrcA HIIrcB HIIrccA HIIrccB HIcic HIcec
 * Brem Compton. */
typedef struct {
	int ar_nrows;
	double ar_min, ar_step_inv;
	const double *ar_logT;
	const double *ar_col[9];
	int xs_nrows;
	double xs_min, xs_step_inv, xs_cut_HI;
	const double *xs_eng;
	const double *xs_HI;
	const double *kernel;           /* 4096 column-depth values */
	int kernel_n;
	double H_PER_MASS, HI_ENERGY, MPROTON_OVER_BOLTZMANN, BOLTZMANN_OVER_MPROTON;
	double hmf, hemf;
	int isothermal, on_the_spot, adiabatic;
} po_tables;

typedef struct po_tree po_tree;

po_tree *po_tree_build(size_t n, const float *pos, const float *sml, double boxsize, int ppc);
void po_tree_free(po_tree *t);
size_t po_tree_ncells(const po_tree *t);
void po_tree_cells(const po_tree *t, int64_t *head, int64_t *first_child, int64_t *parent,
		uint32_t *npar, float *bot, float *top, int64_t *next);
size_t po_tree_skipped(const po_tree *t);

/* One ray: hits (ipar, d, b) sorted by (d, ipar); returns count. *out is
 * grown with realloc as needed (caller frees with po_free). */
size_t po_trace(const po_tree *t, const float *pos, const float *sml, const int8_t *flag,
		const po_ray *ray, po_hit **out, size_t *cap);
void po_free(void *p);

/* Particle state the tick reads and writes (SoA, reference storage types). */
typedef struct {
	size_t n;
	const float *pos, *mass, *sml, *rho, *yeMET;
	const int8_t *flag;
	double *lambdaH;
	float *ie;
	double *yGdepHI;    /* photons absorbed / NH, accumulated in FP64 */
	double *heat;
	int32_t *hits;
	int64_t *lasthit;
} po_state;

typedef struct {
	double total_hits;       /* sum of hit-list lengths (stat.total_deposit_count) */
	double saturated;        /* capped deposits (loop.c:482-485) */
	double active;           /* particles updated */
	double lost_photons;
} po_stats;

/* One full tick (trace, deposit, merge, update) for nray rays.
 * If hits_out is non-NULL it receives, per ray, the sorted hit lists
 * concatenated (offsets[nray+1]). */
int po_tick(const po_tree *t, po_state *st, const po_tables *tb, const po_ray *rays,
		size_t nray, int64_t tick, double tick_time, po_stats *stats);

/* Deposit only: accumulate into st->yGdepHI/heat/hits for the given hit lists. */
int po_deposit(po_state *st, const po_tables *tb, const po_ray *rays, size_t nray,
		const int64_t *offsets, const po_hit *hits, po_stats *stats);

/* Solve one particle step (solve.c:170-224 semantics, own integrator).
 * x = {lambdaH, ie}; returns 0 on success. */
int po_solve(const po_tables *tb, double *lambdaH, double *ie, double yeMET,
		double yGdepHI, double heat, double time, double nH, double T);

int po_solve_numeric(const po_tables *tb, double *lambdaH, double *ie, double yeMET,
		double yGdepHI, double heat, double time, double nH, double T);

double po_ar_get(const po_tables *tb, int col, double logT);
double po_xs_get_HI(const po_tables *tb, double freq);
double po_sph_depth(const po_tables *tb, double r_h);
int po_pluecker(const float dir[3], float dist, const float s2b[3], const float s2t[3]);
#endif
