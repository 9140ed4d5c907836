/* Host-side parts of libpsg: unit system, rate / cross-section / kernel
 * tables. Plain C; each function names the reference code it restates.
 * Compiled without floating-point contraction so every operation rounds once
 * in the written order, as in the reference. */
#include "psg.h"

#include <ctype.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <strings.h>

/* units_init() src/units.c:66-104 */
int psg_units_init(const psg_unit_params *p, psg_units *u) {
	if (!p || !u || p->h <= 0 || p->length_cmh <= 0 || p->mass_gramh <= 0 || p->time_sh <= 0)
		return PSG_E_INVAL;
	memset(u, 0, sizeof(*u));
	const double C_H = p->h;
	u->hmf = p->hmf;
	u->hemf = 1.0 - p->hmf;
	u->CM = C_H / p->length_cmh;
	u->GRAM = C_H / p->mass_gramh;
	u->SEC = C_H / p->time_sh;
	u->M = u->CM * 100;
	u->KM = u->M * 1000;
	u->KPC = u->M * 3.08568025e19;
	u->YR = u->SEC * 31556926.0;
	u->KG = u->GRAM * 1000;
	u->MYR = u->YR * 1e6;
	u->MSUN = u->KG * 1.98892e30;
	u->MPROTON = u->KG * 1.67262158e-27;
	u->KELVIN = 1.0;
	u->BOLTZMANN = 1.3806503e-23 * u->M * u->M * u->KG / u->SEC / u->SEC;
	u->J = u->KG * u->M * u->M / (u->SEC * u->SEC);
	u->EV = 1.602176487e-19 * u->J;
	u->ERG = 1e-7 * u->J;
	u->RY_ENG = 13.60569253 * u->EV;
	u->H_PER_MASS = u->hmf / u->MPROTON;
	u->HE_PER_MASS = u->hemf / (4 * u->MPROTON);
	u->HI_ENERGY = 13.60569253 * u->EV;
	u->HEI_ENERGY = 24.587 * u->EV;
	u->HEII_ENERGY = 54.416 * u->EV;
	u->MPROTON_OVER_BOLTZMANN = u->MPROTON / u->BOLTZMANN;
	u->BOLTZMANN_OVER_MPROTON = 1.0 / (u->MPROTON / u->BOLTZMANN);
	return PSG_OK;
}

/* ---- fixed-width table reader: tabfun_init() src/tabfun.c:60-130 --------
 * '#' lines are comments; then a "min max nrows step" line, a line of
 * 14-character column names, one ignored line, and nrows rows of
 * 14-character fields of which the first 13 characters are read. */
typedef struct {
	int nrows, ncols;
	double min, max, step, step_inv;
	char **names;
	double **data;
} fwtable;

static void fwtable_free(fwtable *t) {
	for (int i = 0; i < t->ncols; i++) {
		free(t->names ? t->names[i] : NULL);
		free(t->data ? t->data[i] : NULL);
	}
	free(t->names);
	free(t->data);
	memset(t, 0, sizeof(*t));
}

static int fwtable_read(const char *path, fwtable *t) {
	memset(t, 0, sizeof(*t));
	FILE *fp = fopen(path, "r");
	if (!fp) return PSG_E_IO;
	char *line = NULL;
	size_t cap = 0;
	ssize_t len;
	int stage = 0, irow = 0, rc = PSG_OK;
	while (stage < 4 && (len = getline(&line, &cap, fp)) >= 0) {
		if (line[0] == '#') continue;
		if (stage == 0) {
			if (sscanf(line, "%lf %lf %d %lf", &t->min, &t->max, &t->nrows, &t->step) != 4
					|| t->nrows < 2 || t->step <= 0) { rc = PSG_E_IO; break; }
			t->step_inv = 1.0 / t->step;
			stage = 1;
		} else if (stage == 1) {
			t->ncols = (int)(len / 14);
			if (t->ncols < 1) { rc = PSG_E_IO; break; }
			t->names = calloc(t->ncols, sizeof(char *));
			t->data = calloc(t->ncols, sizeof(double *));
			for (int i = 0; i < t->ncols; i++) {
				char buf[15];
				memcpy(buf, line + 14 * i, 14);
				buf[14] = 0;
				int e = 13;
				while (e >= 0 && (buf[e] == ' ' || buf[e] == '\n' || buf[e] == '\r')) buf[e--] = 0;
				char *s = buf;
				while (*s == ' ') s++;
				t->names[i] = strdup(s);
				t->data[i] = calloc(t->nrows, sizeof(double));
			}
			stage = 2;
		} else if (stage == 2) {
			stage = 3;
		} else {
			for (int i = 0; i < t->ncols; i++) {
				if (14 * i > len) { rc = PSG_E_IO; break; }
				char buf[14] = {0};
				const ssize_t avail = len - 14 * i;
				memcpy(buf, line + 14 * i, avail < 13 ? (size_t)avail : 13);
				t->data[i][irow] = atof(buf);
			}
			if (rc) break;
			if (++irow == t->nrows) stage = 4;
		}
	}
	free(line);
	fclose(fp);
	if (rc == PSG_OK && stage != 4) rc = PSG_E_IO;
	if (rc) fwtable_free(t);
	return rc;
}

static int fwtable_col(const fwtable *t, const char *name) {
	for (int i = 0; i < t->ncols; i++)
		if (!strcasecmp(name, t->names[i])) return i;
	return -1;
}

/* bremsstrahlung_cen_1992() atomic-rate.c:58-60. The reference evaluates it
 * on the table's first column, which holds log10(T). */
static double brem_fit(double x) { return 1.42e-27 * 1.5 * sqrt(x); }

/* ar_init() atomic-rate.c:66-87 with tabfun_setup_col() tabfun.c:12-36 */
int psg_rate_table_load(const char *path, const psg_units *u, psg_rate_table *out) {
	if (!path || !u || !out) return PSG_E_INVAL;
	memset(out, 0, sizeof(*out));
	fwtable t;
	int rc = fwtable_read(path, &t);
	if (rc) return rc;
	const double rate = u->CM * u->CM * u->CM / u->SEC;
	const double rcool = u->ERG * u->CM * u->CM * u->CM / u->SEC;
	const double coll = u->ERG * (u->CM * u->CM * u->CM) / u->SEC;
	static const char *names[PSG_AR_NCOLS] = {
		"HIci", "HIIrcA", "HIIrcB", "HIIrccA", "HIIrccB", "HIcic", "HIcec", "Brem", "Compton",
		"HeIci", "HeIIci", "HeIIrcA", "HeIIrcB", "HeIIIrcA", "HeIIIrcB"};
	double units[PSG_AR_NCOLS] = {rate, rate, rate, rcool, rcool, coll, coll, coll,
		u->ERG / u->SEC, rate, rate, rate, rate, rate, rate};
	out->nrows = t.nrows;
	out->min = t.min;
	out->max = t.max;
	out->step = t.step;
	out->step_inv = t.step_inv;
	out->logT = malloc(sizeof(double) * t.nrows);
	memcpy(out->logT, t.data[0], sizeof(double) * t.nrows);
	for (int c = 0; c < PSG_AR_NCOLS; c++) {
		out->col[c] = malloc(sizeof(double) * t.nrows);
		const int k = fwtable_col(&t, names[c]);
		if (k >= 0) {
			for (int j = 0; j < t.nrows; j++) out->col[c][j] = t.data[k][j] * units[c];
		} else if (c == PSG_AR_E_BREMC) {
			for (int j = 0; j < t.nrows; j++) out->col[c][j] = brem_fit(t.data[0][j]) * units[c];
		} else if (c == PSG_AR_E_COMPC) {
			for (int j = 0; j < t.nrows; j++) out->col[c][j] = 0.0 * units[c];
		} else {
			rc = PSG_E_IO;     /* the reference stops: "column unknown" */
		}
	}
	fwtable_free(&t);
	if (rc) psg_rate_table_free(out);
	return rc;
}

void psg_rate_table_free(psg_rate_table *t) {
	if (!t) return;
	free(t->logT);
	for (int c = 0; c < PSG_AR_NCOLS; c++) free(t->col[c]);
	memset(t, 0, sizeof(*t));
}

/* tabfun_get() tabfun.c:38-58: linear in the uniform grid; the index is the
 * truncated (value-min)/step, so values just below min extrapolate from the
 * first interval and anything past it clamps to an end row. */
static double tab_get(int nrows, double min, double step_inv, const double *x, const double *y,
		double v) {
	const long idx = (long)((v - min) * step_inv);
	if (idx < 0) return y[0];
	if (idx >= nrows - 1) return y[nrows - 1];
	const double lw = x[idx + 1] - v;
	const double rw = v - x[idx];
	return (lw * y[idx] + rw * y[idx + 1]) * step_inv;
}

double psg_ar_get(const psg_rate_table *t, int col, double logT) {
	return tab_get(t->nrows, t->min, t->step_inv, t->logT, t->col[col], logT);
}

/* ---- photo-ionisation cross sections, src/verner.F90 (single-precision
 * Fortran functions; a `real` meeting a d0 literal is promoted to double and
 * rounded back to float on assignment). */
static float sigma_HI_verner(float Ry) {
	const float E0 = 4.298e-1f, sig0 = 5.475e4f, ya = 3.288e1f, P = 2.963f;
	if (Ry < 0.5f) return 0.0f;
	const float eV = (float)((double)Ry * 13.6);
	const float x = eV / E0;
	const float y = x;
	const float xm1 = x - 1.0f;
	const float a = sig0 * (xm1 * xm1);
	const double e = 0.5 * (double)P - 5.5;
	const double b = (double)a * pow((double)y, e);
	const float c = powf(1.0f + sqrtf(y / ya), -P);
	float s = (float)(b * (double)c);
	s = (float)((double)s * 1.0e-18);
	return s < 0.0f ? 0.0f : s;
}
static float sigma_HeI_osterbrock(float Ry) {
	const float nu = 24.587f;
	if (2.0f * Ry * 13.6f < nu) return 0.0f;
	const float sf = Ry * 13.6f / nu;
	return 7.2e-18f * (1.66f * powf(sf, -2.05f) + 0.66f * powf(sf, -3.05f));
}
static float sigma_HeII_osterbrock(float Ry) {
	const float nu = 54.416f;
	if (2.0f * Ry * 13.6f < nu) return 0.0f;
	const float s = Ry * 13.6f / nu;
	return 1.58e-18f * (1.0f / (s * s * s));
}

/* xs_init(NULL) atomic-rate.c:93-124 */
int psg_xs_table_build(const psg_units *u, psg_xs_table *t) {
	if (!u || !t) return PSG_E_INVAL;
	memset(t, 0, sizeof(*t));
	t->nrows = 16384;
	t->min = 1 * u->HI_ENERGY;
	t->max = 100 * u->HI_ENERGY;
	t->step = (t->max - t->min) / (t->nrows - 1);
	t->step_inv = 1.0 / t->step;
	t->eng = malloc(sizeof(double) * t->nrows);
	for (int s = 0; s < PSG_XS_NSPECIES; s++) t->sigma[s] = malloc(sizeof(double) * t->nrows);
	const double cm2 = u->CM * u->CM;
	for (int i = 0; i < t->nrows; i++) {
		const double eng = t->min + t->step * i;
		t->eng[i] = eng;
		const float ryd = (float)(eng / u->HI_ENERGY);
		t->sigma[PSG_XS_HI][i] = (double)sigma_HI_verner(ryd) * cm2;
		t->sigma[PSG_XS_HEI][i] = (double)sigma_HeI_osterbrock(ryd) * cm2;
		t->sigma[PSG_XS_HEII][i] = (double)sigma_HeII_osterbrock(ryd) * cm2;
	}
	/* the deliberate low cuts of atomic-rate.c:117-122 */
	t->cut[PSG_XS_HI] = 13.6 * u->EV;
	t->cut[PSG_XS_HEI] = 24.5 * u->EV;
	t->cut[PSG_XS_HEII] = 54.4 * u->EV;
	return PSG_OK;
}

void psg_xs_table_free(psg_xs_table *t) {
	if (!t) return;
	free(t->eng);
	for (int s = 0; s < PSG_XS_NSPECIES; s++) free(t->sigma[s]);
	memset(t, 0, sizeof(*t));
}

double psg_xs_get(const psg_xs_table *t, int species, double freq) {
	if (freq < t->cut[species]) return 0.0;
	return tab_get(t->nrows, t->min, t->step_inv, t->eng, t->sigma[species], freq);
}

/* ---- secondary ionisation: secion.c -------------------------------------- */
/* The fits of Ricotti, Gnedin & Shull (2002, ApJ 575, 33) as secion.c
 * writes them: for the ionisation fractions (k = 0 HI, 1 HeI)
 *     Phi = A_k (1 - x^b_k)^c_k [E >= E_0 - 0.1]
 *         - A'_k x^0.2 (1 - x^0.38)^2 [E >= E_0 - 0.1] (E_0/E)^0.4,  E_0 = 28 eV,
 * and for the heating fraction
 *     Eh = 1 - (1 - x^0.2663)^1.3163 [E >= E_1 - 0.1]
 *        + 3.9811 x^0.4 (1 - x^0.34)^2 [E >= E_1 - 0.1] (E_1/E)^0.7,  E_1 = 11 eV
 * (the 0.1 is subtracted in internal energy units, as there). */
static const double RGS_A[2] = {0.3908, 0.0554}, RGS_B[2] = {0.4092, 0.4614}, RGS_C[2] = {1.7592, 1.6660};
static const double RGS_A2[2] = {0.6941, 0.0984};

static double rgs_phi(int k, double E, double x, double ev) {
	const double gate = 28 * ev;
	const int f1 = (E >= (gate - 0.1));
	const double f2 = f1 * pow(gate / E, 0.4);
	const double y1 = RGS_A[k] * pow(1. - pow(x, RGS_B[k]), RGS_C[k]);
	const double y2 = RGS_A2[k] * pow(x, 0.2) * pow(1 - pow(x, 0.38), 2.0);
	return (y1 * f1 - y2 * f2);
}

static double rgs_heat(double E, double x, double ev) {
	const double gate = 11 * ev;
	const int f1 = (E >= gate - 0.1);
	const double f2 = f1 * pow(gate / E, 0.7);
	const double y1 = 1.0 * pow(1 - pow(x, 0.2663), 1.3163);
	const double y2 = 3.9811 * pow(x, 0.4) * pow(1 - pow(x, 0.34), 2.0);
	return (1. - y1 * f1 + y2 * f2);
}

/* secion_init() secion.c:74-98 with tabfun2_ensure_col() tabfun.c:151-171 */
int psg_secion_table_build(const psg_units *u, double *out) {
	if (!u || !out) return PSG_E_INVAL;
	const double min1 = 10 * u->EV, max1 = 200 * u->EV, min2 = -8, max2 = 0;
	const double step1 = (max1 - min1) / PSG_SECION_NE, step2 = (max2 - min2) / PSG_SECION_NX;
	const size_t plane = (size_t)PSG_SECION_NE * PSG_SECION_NX;
	for (int i = 0; i < PSG_SECION_NE; i++) {
		const double E = min1 + i * step1;
		for (int j = 0; j < PSG_SECION_NX; j++) {
			const double x = pow(10, min2 + j * step2);
			const size_t o = (size_t)i * PSG_SECION_NX + j;
			out[o] = rgs_phi(0, E, x, u->EV);
			out[plane + o] = rgs_phi(1, E, x, u->EV);
			out[2 * plane + o] = rgs_heat(E, x, u->EV);
		}
	}
	return PSG_OK;
}

/* ---- kernel.akline reader and sph_depth() sph-depth.c:26-33 ------------- */
int psg_kernel_table_load(const char *path, double *out, int cap, int *n) {
	if (!path || !out || !n || cap <= 0) return PSG_E_INVAL;
	FILE *fp = fopen(path, "r");
	if (!fp) return PSG_E_IO;
	char buf[256];
	int k = 0, rc = PSG_OK;
	while (fgets(buf, sizeof(buf), fp)) {
		char *s = buf;
		while (isspace((unsigned char)*s)) s++;
		if (!*s) continue;
		char *end = NULL;
		const double v = strtod(s, &end);
		if (end == s) { rc = PSG_E_IO; break; }
		if (k == cap) { rc = PSG_E_OVERFLOW; break; }
		out[k++] = v;
	}
	fclose(fp);
	*n = k;
	if (rc == PSG_OK && k == 0) rc = PSG_E_IO;
	return rc;
}

double psg_sph_depth(const double *table, int n, double r_h) {
	const int i = (int)(n * r_h);
	if (i < n && i >= 0) return table[i];
	return 0.0;
}
