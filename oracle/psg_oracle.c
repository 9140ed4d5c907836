/* CPU restatement of psphray's trace -> deposit -> merge -> update hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker for the CUDA path; the product never
 * links it). Parity of this restatement is pinned against the reference's own
 * code compiled into oracle/_ref/libpsphray_ref.so, in tests/.
 *
 * Built with -ffp-contract=off so that every float/double operation rounds
 * exactly once, in the order written, as in the reference. */
#include "psg_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* Octree, restating rt_switch_epoch() raytrace.c:41-151 and its helpers
 * inside/find/split/add/full raytrace.c:232-317: a region octree over
 * [0, boxsize)^3, children numbered by bit d = upper half along axis d, a leaf
 * splits when a particle arrives while it already holds ppc particles, and
 * afterwards every cell's box becomes the AABB of pos +- sml of its particles
 * (leaves) or of its 8 children (internal cells); an empty leaf keeps its
 * region box. */
struct po_tree {
	size_t ncell, cap;
	float (*bot)[3], (*top)[3];
	int64_t *head, *first_child, *parent;
	uint32_t *npar;
	int64_t *next;
	size_t n, skipped;
};

static int64_t new_cells(po_tree *t, int count) {
	if (t->ncell + count > t->cap) {
		size_t c = t->cap ? t->cap * 2 : 1024;
		while (c < t->ncell + count) c *= 2;
		t->bot = realloc(t->bot, c * sizeof(*t->bot));
		t->top = realloc(t->top, c * sizeof(*t->top));
		t->head = realloc(t->head, c * sizeof(int64_t));
		t->first_child = realloc(t->first_child, c * sizeof(int64_t));
		t->parent = realloc(t->parent, c * sizeof(int64_t));
		t->npar = realloc(t->npar, c * sizeof(uint32_t));
		t->cap = c;
	}
	int64_t first = (int64_t)t->ncell;
	t->ncell += count;
	return first;
}

static int in_region(const po_tree *t, const float *p, int64_t c) {
	for (int d = 0; d < 3; d++)
		if (p[d] >= t->top[c][d] || p[d] < t->bot[c][d]) return 0;
	return 1;
}

static int64_t descend(const po_tree *t, const float *p, int64_t c) {
	while (t->first_child[c] != -1) {
		int64_t fc = t->first_child[c], k;
		for (k = 0; k < 8; k++)
			if (in_region(t, p, fc + k)) break;
		c = fc + k;     /* in_region of the parent guarantees one child matches */
	}
	return c;
}

static void leaf_push(po_tree *t, int64_t ipar, int64_t c) {
	t->next[ipar] = t->head[c];
	t->head[c] = ipar;
	t->npar[c]++;
}

static void split_leaf(po_tree *t, const float *pos, int64_t c) {
	int64_t fc = new_cells(t, 8);
	float mid[3];
	for (int d = 0; d < 3; d++) {
		const float sum = t->top[c][d] + t->bot[c][d];   /* float add, then halve */
		mid[d] = (float)(0.5 * sum);
	}
	for (int k = 0; k < 8; k++) {
		for (int d = 0; d < 3; d++) {
			const int upper = (k >> d) & 1;
			t->bot[fc + k][d] = upper ? mid[d] : t->bot[c][d];
			t->top[fc + k][d] = upper ? t->top[c][d] : mid[d];
		}
		t->parent[fc + k] = c;
		t->first_child[fc + k] = -1;
		t->head[fc + k] = -1;
		t->npar[fc + k] = 0;
	}
	t->first_child[c] = fc;
	int64_t p = t->head[c];
	t->head[c] = -1;
	t->npar[c] = 0;
	while (p != -1) {
		int64_t nx = t->next[p];
		for (int k = 0; k < 8; k++)
			if (in_region(t, pos + 3 * p, fc + k)) { leaf_push(t, p, fc + k); break; }
		p = nx;
	}
}

po_tree *po_tree_build(size_t n, const float *pos, const float *sml, double boxsize, int ppc) {
	po_tree *t = calloc(1, sizeof(po_tree));
	t->n = n;
	t->next = malloc(n * sizeof(int64_t));
	for (size_t i = 0; i < n; i++) t->next[i] = -1;
	new_cells(t, 1);
	for (int d = 0; d < 3; d++) { t->bot[0][d] = 0; t->top[0][d] = (float)boxsize; }
	t->parent[0] = -1; t->first_child[0] = -1; t->head[0] = -1; t->npar[0] = 0;
	for (size_t i = 0; i < n; i++) {
		const float *p = pos + 3 * i;
		if (!in_region(t, p, 0)) { t->skipped++; continue; }
		int64_t c = descend(t, p, 0);
		while (t->npar[c] >= (uint32_t)ppc) {
			split_leaf(t, pos, c);
			c = descend(t, p, c);
		}
		leaf_push(t, (int64_t)i, c);
	}
	/* AABB pass: children are always allocated after their parent, so a
	 * reverse sweep finishes every child before its parent. */
	for (int64_t c = (int64_t)t->ncell - 1; c >= 0; c--) {
		float *bo = t->bot[c], *to = t->top[c];
		if (t->first_child[c] == -1) {
			int first = 1;
			for (int64_t p = t->head[c]; p != -1; p = t->next[p]) {
				for (int d = 0; d < 3; d++) {
					const float lo = pos[3 * p + d] - sml[p];
					const float hi = pos[3 * p + d] + sml[p];
					if (first || lo < bo[d]) bo[d] = lo;
					if (first || hi > to[d]) to[d] = hi;
				}
				first = 0;
			}
		} else {
			const int64_t fc = t->first_child[c];
			for (int k = 0; k < 8; k++)
				for (int d = 0; d < 3; d++) {
					if (k == 0 || t->bot[fc + k][d] < bo[d]) bo[d] = t->bot[fc + k][d];
					if (k == 0 || t->top[fc + k][d] > to[d]) to[d] = t->top[fc + k][d];
				}
		}
	}
	return t;
}

void po_tree_free(po_tree *t) {
	if (!t) return;
	free(t->bot); free(t->top); free(t->head); free(t->first_child);
	free(t->parent); free(t->npar); free(t->next); free(t);
}
size_t po_tree_ncells(const po_tree *t) { return t->ncell; }
size_t po_tree_skipped(const po_tree *t) { return t->skipped; }
void po_tree_cells(const po_tree *t, int64_t *head, int64_t *first_child, int64_t *parent,
		uint32_t *npar, float *bot, float *top, int64_t *next) {
	for (size_t c = 0; c < t->ncell; c++) {
		head[c] = t->head[c]; first_child[c] = t->first_child[c];
		parent[c] = t->parent[c]; npar[c] = t->npar[c];
		for (int d = 0; d < 3; d++) { bot[3 * c + d] = t->bot[c][d]; top[3 * c + d] = t->top[c][d]; }
	}
	for (size_t i = 0; i < t->n; i++) next[i] = t->next[i];
}

/* ------------------------------------------------------------------------ */
/* Segment-vs-box test, restating pluecker_() pluecker-sse.c:28-198.
 * The reference spells out 8 direction-sign classes; they all reduce to one
 * rule per axis and per axis pair, written here with selects:
 *   axis a moving up (dir>0): reject if box top is below the start or the
 *   box bottom is above the end; moving down: the mirror image.
 *   pair (i,j): with P,R picked by the sign of dir[i] and Q,S by the sign of
 *   dir[j], reject if dir[i]*P < dir[j]*Q or dir[i]*R > dir[j]*S.
 * Every product and difference is a single float rounding. */
int po_pluecker(const float dir[3], float dist, const float s2b[3], const float s2t[3]) {
	float e2b[3], e2t[3];
	int up[3];
	for (int a = 0; a < 3; a++) {
		const float step = dist * dir[a];
		e2t[a] = s2t[a] - step;
		e2b[a] = s2b[a] - step;
		up[a] = dir[a] > 0;
	}
	for (int a = 0; a < 3; a++) {
		if (up[a] ? (s2t[a] < 0) : (s2b[a] > 0)) return 0;
		if (up[a] ? (e2b[a] > 0) : (e2t[a] < 0)) return 0;
	}
	static const int pi[3] = {0, 0, 1}, pj[3] = {1, 2, 2};
	for (int q = 0; q < 3; q++) {
		const int i = pi[q], j = pj[q];
		const float P = up[i] ? s2t[j] : s2b[j];
		const float R = up[i] ? s2b[j] : s2t[j];
		const float Q = up[j] ? s2b[i] : s2t[i];
		const float S = up[j] ? s2t[i] : s2b[i];
		const float r0 = dir[i] * P, r1 = dir[j] * Q, r2 = dir[i] * R, r3 = dir[j] * S;
		if (r0 < r1 || r2 > r3) return 0;
	}
	return 1;
}

static int hit_cell(const po_tree *t, const float *s, const float *dir, float dist, int64_t c) {
	float s2b[3], s2t[3];
	for (int d = 0; d < 3; d++) {
		s2b[d] = t->bot[c][d] - s[d];
		s2t[d] = t->top[c][d] - s[d];
	}
	return po_pluecker(dir, dist, s2b, s2t);
}

static int hit_cmp(const void *a, const void *b) {
	const po_hit *x = a, *y = b;
	if (x->d < y->d) return -1;
	if (x->d > y->d) return 1;
	return (x->ipar > y->ipar) - (x->ipar < y->ipar);
}

/* rt_trace() raytrace.c:153-210: walk cells depth first (children 0..7),
 * descend only into cells whose box the segment [s, s + dist*dir] crosses,
 * and in each crossed leaf accept every particle whose smoothing sphere the
 * ray's line passes through (raytrace.c:168-195: float differences, float
 * products, double sums; d is the distance to the centre). Then the per-ray
 * sort of loop.c:383, with ties in d broken by particle index. */
size_t po_trace(const po_tree *t, const float *pos, const float *sml, const int8_t *flag,
		const po_ray *ray, po_hit **out, size_t *cap) {
	const float dist = (float)ray->length;
	const float *s = ray->s, *dir = ray->dir;
	size_t len = 0;
	int64_t c = 0;
	while (c != -1) {
		if (hit_cell(t, s, dir, dist, c)) {
			if (t->first_child[c] != -1) { c = t->first_child[c]; continue; }
			for (int64_t p = t->head[c]; p != -1; p = t->next[p]) {
				if (flag && (flag[p] & 1)) continue;
				/* raytrace.c:176-183 as the reference's build runs it: float
				 * differences and products; the double sums reassociated
				 * by its -O3 -ffast-math into (y + z) + x (the order of
				 * its compiled x86 code), not the source's x, y, z */
				float pr[3], sq[3];
				for (int d = 0; d < 3; d++) {
					const float dd = pos[3 * p + d] - s[d];
					pr[d] = dd * dir[d];
					sq[d] = dd * dd;
				}
				const double proj = ((double)pr[1] + (double)pr[2]) + (double)pr[0];
				const double dd2 = ((double)sq[1] + (double)sq[2]) + (double)sq[0];
				const double dc = sqrt(dd2);
				const double r2 = (dc - proj) * (dc + proj);
				const float h2 = sml[p] * sml[p];
				if (h2 < r2) continue;
				if (len == *cap) {
					*cap = *cap ? *cap * 2 : 1024;
					*out = realloc(*out, *cap * sizeof(po_hit));
				}
				(*out)[len].ipar = p;
				(*out)[len].d = dc;
				(*out)[len].b = sqrt(fabs(r2));
				len++;
			}
		}
		/* next cell: the next sibling, else the next sibling of an ancestor */
		int64_t nx = -1;
		while (c != 0) {
			const int64_t par = t->parent[c];
			if (c - t->first_child[par] != 7) { nx = c + 1; break; }
			c = par;
		}
		c = nx;
	}
	qsort(*out, len, sizeof(po_hit), hit_cmp);
	return len;
}

void po_free(void *p) { free(p); }

/* ------------------------------------------------------------------------ */
/* Tables: tabfun_get() tabfun.c:38-58 (linear in a uniform grid, clamped to
 * the end rows), xs_get() atomic-rate.c:126-131 (zero below the cut),
 * sph_depth() sph-depth.c:26-33 (truncated index, zero outside). */
static double tab_lookup(int nrows, double min, double step_inv, const double *x,
		const double *y, double v) {
	const long idx = (long)((v - min) * step_inv);
	if (idx < 0) return y[0];
	if (idx >= nrows - 1) return y[nrows - 1];
	const double lw = x[idx + 1] - v;
	const double rw = v - x[idx];
	return (lw * y[idx] + rw * y[idx + 1]) * step_inv;
}

double po_ar_get(const po_tables *tb, int col, double logT) {
	return tab_lookup(tb->ar_nrows, tb->ar_min, tb->ar_step_inv, tb->ar_logT, tb->ar_col[col], logT);
}

double po_xs_get_HI(const po_tables *tb, double freq) {
	if (freq < tb->xs_cut_HI) return 0.0;
	return tab_lookup(tb->xs_nrows, tb->xs_min, tb->xs_step_inv, tb->xs_eng, tb->xs_HI, freq);
}

double po_sph_depth(const po_tables *tb, double r_h) {
	const int n = (int)(tb->kernel_n * r_h);
	if (n < tb->kernel_n && n >= 0) return tb->kernel[n];
	return 0.0;
}

/* ------------------------------------------------------------------------ */
/* deposit() loop.c:388-608, hydrogen-only branch without EOS, comoving
 * scaling or secondary ionisation: walk each ray's sorted hits, optical depth
 * tau = sigma * kernel * xHI * NH, absorb TM*(1-e^-tau) capped at the
 * particle's neutral atoms, stop once TM/Nph < 1e-10. Per-particle sums are
 * FP64 here (the reference adds into float with omp atomics). */
static void deposit_ray(po_state *st, const po_tables *tb, const po_ray *ray,
		const po_hit *x, size_t nx, po_stats *stats) {
	if (nx == 0 || ray->Nph == 0) return;
	double TM = ray->Nph;
	const double sigmaHI = po_xs_get_HI(tb, ray->freq);
	const double dEHI = fdim(ray->freq, tb->HI_ENERGY);
	const double heat_factor_HI = tb->H_PER_MASS * dEHI;
	for (size_t j = 0; j < nx; j++) {
		const int64_t p = x[j].ipar;
		const double b = x[j].b;
		const double sml = st->sml[p];
		const double sml_inv = 1.0 / sml;
		const double NH = (double)st->mass[p] * tb->H_PER_MASS;
		const double NH_inv = 1.0 / NH;
		const double xHI = st->lambdaH[p];
		const double kernel = po_sph_depth(tb, b * sml_inv) * (sml_inv * sml_inv);
		const double NHI = xHI * NH;
		const double tau = sigmaHI * (kernel * NHI);
		if (tau == 0.0) continue;
		double absorb = -TM * expm1(-tau);
		if (absorb > NHI) {
			absorb = NHI;
			if (stats) stats->saturated += 1;
		}
		const double delta = absorb * NH_inv;
		st->yGdepHI[p] += delta;
		st->heat[p] += heat_factor_HI * delta;
		st->hits[p] += 1;
		TM -= absorb;
		if (TM < 0.0 || TM / ray->Nph < 1e-10) break;
	}
	if (stats) stats->lost_photons += TM;
}

int po_deposit(po_state *st, const po_tables *tb, const po_ray *rays, size_t nray,
		const int64_t *offsets, const po_hit *hits, po_stats *stats) {
	for (size_t i = 0; i < nray; i++) {
		const size_t nx = (size_t)(offsets[i + 1] - offsets[i]);
		if (stats) stats->total_hits += (double)nx;
		deposit_ray(st, tb, &rays[i], hits + offsets[i], nx, stats);
	}
	return 0;
}

/* ------------------------------------------------------------------------ */
/* Solver. The reference integrates the 7-variable system of solve.c:76-141
 * over normalised time s in [0,1] with LSODA (solve.c:170-224). In the
 * hydrogen-only, on-the-spot case only lambdaH (and ie when not isothermal)
 * move; the others have zero derivative.
 *
 * Isothermal: with ye = 1 + m - lambda (m = yeMET plus the frozen helium
 * electrons) the equation d(lambda)/ds = -g + tau*ye*(alpha*(1-lambda) -
 * gamma*lambda) is a Riccati equation with constant coefficients,
 *     d(lambda)/ds = a*lambda^2 - b*lambda + c,
 * solved in closed form about its stable root p1 (y = lambda - p1):
 *     y(1) = y0*E / (1 - a*y0*phi(k)),  k = sqrt(b^2-4ac), E = e^-k,
 *     phi(k) = (1 - e^-k)/k,
 * where b^2-4ac = q^2 + 4*a*g with q = tau*(gamma*(1+m) + alpha*m) >= 0 is
 * evaluated without cancellation and p1 = 2c/(b + k).
 *
 * Not isothermal: lambda and ie integrated together with an adaptive
 * Dormand-Prince 5(4) method at tight tolerance (an accuracy reference, not
 * a restatement of LSODA's steps). */
enum { AR_HI_CI, AR_HII_RC_A, AR_HII_RC_B, AR_HII_RCC_A, AR_HII_RCC_B, AR_HI_CIC, AR_HI_CEC, AR_BREM, AR_COMPTON };

static double ieye2T(const po_tables *tb, double ie, double ye) {
	return tb->MPROTON_OVER_BOLTZMANN * ie / (tb->hemf * 0.25 + tb->hmf + tb->hmf * ye) * 2.0 / 3.0;
}
static double Tye2ie(const po_tables *tb, double T, double ye) {
	return T * tb->BOLTZMANN_OVER_MPROTON * (tb->hemf * 0.25 + tb->hmf + tb->hmf * ye) / 2.0 * 3.0;
}
/* helium electrons per hydrogen with helium frozen neutral-less as the
 * hydrogen-only run leaves it (lambdaHeI = lambdaHeII = 0 => xHeIII = 1),
 * psystem.h:134-137 */
static double he_electrons(const po_tables *tb) {
	return tb->hemf / tb->hmf * 0.25 * (0.0 + 2 * (1.0 - 0.0 - 0.0));
}

static double phi_k(double k) {
	if (k > 1e-6) return -expm1(-k) / k;
	return 1.0 - k * (0.5 - k / 6.0);
}

static double riccati_step(double lam0, double a, double b, double q, double c, double g) {
	if (!(a > 0.0)) {
		/* linear limit: d(lambda)/ds = -b*lambda + c */
		if (b > 0.0) {
			const double eq = c / b;
			return eq + (lam0 - eq) * exp(-b);
		}
		return lam0 + c;
	}
	const double k = sqrt(q * q + 4.0 * a * g);
	const double p1 = 2.0 * c / (b + k);
	const double y0 = lam0 - p1;
	const double y1 = y0 * exp(-k) / (1.0 - a * y0 * phi_k(k));
	return p1 + y1;
}

typedef struct {
	const po_tables *tb;
	double yeMET, g, heat, time, nH, T;
} rhs_ctx;

static void rhs(const rhs_ctx *cx, const double *x, double *dx) {
	const po_tables *tb = cx->tb;
	const double xHI = x[0], xHII = 1.0 - x[0];
	const double ye = xHII + he_electrons(tb) + cx->yeMET;
	const double T = tb->isothermal ? cx->T : ieye2T(tb, x[1], ye);
	const double logT = log10(T);
	const double nH = cx->nH;
	const double gamma_HI = po_ar_get(tb, AR_HI_CI, logT) * nH;
	const double alpha_A = po_ar_get(tb, AR_HII_RC_A, logT) * nH;
	const double alpha_B = po_ar_get(tb, AR_HII_RC_B, logT) * nH;
	const double alpha = tb->on_the_spot ? alpha_B : alpha_A;
	dx[0] = -cx->g / cx->time + (-gamma_HI * ye * xHI + alpha * ye * xHII);
	if (tb->isothermal || tb->adiabatic) {
		dx[1] = 0.0;
	} else {
		const double eta = po_ar_get(tb, tb->on_the_spot ? AR_HII_RCC_B : AR_HII_RCC_A, logT) * nH;
		const double psi = po_ar_get(tb, AR_HI_CEC, logT) * nH;
		const double zeta = po_ar_get(tb, AR_HI_CIC, logT) * nH;
		const double beta = po_ar_get(tb, AR_BREM, logT) * nH;
		const double chi = po_ar_get(tb, AR_COMPTON, logT);
		const double L = tb->H_PER_MASS * ((zeta + psi) * ye * xHI + eta * ye * xHII
				+ beta * ye * xHII + chi * ye);
		dx[1] = cx->heat / cx->time - L;
	}
	dx[0] *= cx->time;
	dx[1] *= cx->time;
}

static int dopri_integrate(const rhs_ctx *cx, double *x) {
	static const double c2 = 1. / 5, c3 = 3. / 10, c4 = 4. / 5, c5 = 8. / 9;
	static const double a21 = 1. / 5;
	static const double a31 = 3. / 40, a32 = 9. / 40;
	static const double a41 = 44. / 45, a42 = -56. / 15, a43 = 32. / 9;
	static const double a51 = 19372. / 6561, a52 = -25360. / 2187, a53 = 64448. / 6561, a54 = -212. / 729;
	static const double a61 = 9017. / 3168, a62 = -355. / 33, a63 = 46732. / 5247, a64 = 49. / 176, a65 = -5103. / 18656;
	static const double b1 = 35. / 384, b3 = 500. / 1113, b4 = 125. / 192, b5 = -2187. / 6784, b6 = 11. / 84;
	static const double e1 = 71. / 57600, e3 = -71. / 16695, e4 = 71. / 1920, e5 = -17253. / 339200, e6 = 22. / 525, e7 = -1. / 40;
	(void)c2; (void)c3; (void)c4; (void)c5;
	const double rtol = 1e-10, atol[2] = {1e-14, 1e-12 * fabs(x[1]) + 1e-30};
	double t = 0.0, h = 1e-4;
	double k1[2], k2[2], k3[2], k4[2], k5[2], k6[2], k7[2], y[2], yn[2];
	rhs(cx, x, k1);
	for (long it = 0; it < 20000000 && t < 1.0; it++) {
		if (t + h > 1.0) h = 1.0 - t;
		for (int i = 0; i < 2; i++) y[i] = x[i] + h * (a21 * k1[i]);
		rhs(cx, y, k2);
		for (int i = 0; i < 2; i++) y[i] = x[i] + h * (a31 * k1[i] + a32 * k2[i]);
		rhs(cx, y, k3);
		for (int i = 0; i < 2; i++) y[i] = x[i] + h * (a41 * k1[i] + a42 * k2[i] + a43 * k3[i]);
		rhs(cx, y, k4);
		for (int i = 0; i < 2; i++) y[i] = x[i] + h * (a51 * k1[i] + a52 * k2[i] + a53 * k3[i] + a54 * k4[i]);
		rhs(cx, y, k5);
		for (int i = 0; i < 2; i++) y[i] = x[i] + h * (a61 * k1[i] + a62 * k2[i] + a63 * k3[i] + a64 * k4[i] + a65 * k5[i]);
		rhs(cx, y, k6);
		for (int i = 0; i < 2; i++) yn[i] = x[i] + h * (b1 * k1[i] + b3 * k3[i] + b4 * k4[i] + b5 * k5[i] + b6 * k6[i]);
		rhs(cx, yn, k7);
		double err = 0.0;
		for (int i = 0; i < 2; i++) {
			const double e = h * (e1 * k1[i] + e3 * k3[i] + e4 * k4[i] + e5 * k5[i] + e6 * k6[i] + e7 * k7[i]);
			const double sc = atol[i] + rtol * fmax(fabs(x[i]), fabs(yn[i]));
			const double r = e / sc;
			err += r * r;
		}
		err = sqrt(err / 2);
		if (err <= 1.0) {
			t += h;
			x[0] = yn[0]; x[1] = yn[1];
			k1[0] = k7[0]; k1[1] = k7[1];
		}
		double fac = err > 0 ? 0.9 * pow(err, -0.2) : 5.0;
		if (fac > 5.0) fac = 5.0;
		if (fac < 0.2) fac = 0.2;
		h *= fac;
		if (h < 1e-14) h = 1e-14;
	}
	return t < 1.0 ? -1 : 0;
}

/* The same step integrated numerically (Dormand-Prince at rtol 1e-10) even
 * when isothermal: an accuracy check of the closed form. */
int po_solve_numeric(const po_tables *tb, double *lambdaH, double *ie, double yeMET,
		double g, double heat, double time, double nH, double T) {
	rhs_ctx cx = {tb, yeMET, g, heat, time, nH, T};
	double x[2] = {*lambdaH, *ie};
	const int rc = dopri_integrate(&cx, x);
	*lambdaH = fmin(1.0, fmax(0.0, x[0]));
	*ie = x[1];
	return rc;
}

int po_solve(const po_tables *tb, double *lambdaH, double *ie, double yeMET,
		double g, double heat, double time, double nH, double T) {
	int rc = 0;
	if (tb->isothermal) {
		const double logT = log10(T);
		const double gamma = po_ar_get(tb, AR_HI_CI, logT) * nH;
		const double alpha = po_ar_get(tb, tb->on_the_spot ? AR_HII_RC_B : AR_HII_RC_A, logT) * nH;
		const double m = yeMET + he_electrons(tb);
		const double a = time * (alpha + gamma);
		const double b = time * (alpha + (alpha + gamma) * (1.0 + m));
		const double q = time * (gamma * (1.0 + m) + alpha * m);
		const double c = time * alpha * (1.0 + m) - g;
		*lambdaH = riccati_step(*lambdaH, a, b, q, c, g);
	} else {
		rhs_ctx cx = {tb, yeMET, g, heat, time, nH, T};
		double x[2] = {*lambdaH, *ie};
		rc = dopri_integrate(&cx, x);
		*lambdaH = x[0];
		*ie = x[1];
	}
	*lambdaH = fmin(1.0, fmax(0.0, *lambdaH));
	return rc;
}

/* update_pars() loop.c:647-776 for one particle. */
static int update_particle(po_state *st, const po_tables *tb, int64_t p, int64_t tick, double tick_time) {
	const double rho = st->rho[p];
	const double time = (double)(tick - st->lasthit[p]) * tick_time;
	const double ye0 = (1.0 - st->lambdaH[p]) + he_electrons(tb);
	const double T = ieye2T(tb, (double)st->ie[p], ye0);
	double lam = st->lambdaH[p];
	double ie = st->ie[p];
	const double nH = tb->H_PER_MASS * rho;
	const int rc = po_solve(tb, &lam, &ie, (double)st->yeMET[p], st->yGdepHI[p], st->heat[p],
			time, nH, T);
	st->yGdepHI[p] = 0.0;      /* times step_remain, which LSODA leaves at 0 */
	st->lambdaH[p] = lam;
	if (!tb->adiabatic) st->ie[p] = (float)ie;
	st->lasthit[p] = tick;
	if (tb->isothermal) {
		const double ye1 = (1.0 - lam) + he_electrons(tb);
		st->ie[p] = (float)Tye2ie(tb, T, ye1);
	}
	st->heat[p] = 0.0;
	return rc;
}

int po_tick(const po_tree *t, po_state *st, const po_tables *tb, const po_ray *rays,
		size_t nray, int64_t tick, double tick_time, po_stats *stats) {
	po_hit *buf = NULL;
	size_t cap = 0;
	int64_t *off = malloc((nray + 1) * sizeof(int64_t));
	po_hit *all = NULL;
	size_t total = 0, allcap = 0;
	off[0] = 0;
	for (size_t i = 0; i < nray; i++) {
		size_t nx = po_trace(t, st->pos, st->sml, st->flag, &rays[i], &buf, &cap);
		if (total + nx > allcap) {
			allcap = (total + nx) * 2 + 1024;
			all = realloc(all, allcap * sizeof(po_hit));
		}
		memcpy(all + total, buf, nx * sizeof(po_hit));
		total += nx;
		off[i + 1] = (int64_t)total;
	}
	po_deposit(st, tb, rays, nray, off, all, stats);
	/* merge_pars() loop.c:610-645: unique hit particles (every traced hit,
	 * deposited or not), then update each once. */
	uint8_t *seen = calloc(st->n, 1);
	int rc = 0;
	for (size_t h = 0; h < total; h++) {
		const int64_t p = all[h].ipar;
		if (seen[p]) continue;
		seen[p] = 1;
		if (stats) stats->active += 1;
		rc |= update_particle(st, tb, p, tick, tick_time);
	}
	free(seen); free(all); free(off); free(buf);
	return rc;
}
