/* Oracle harness around the reference's own CPU code.
 *
 * This translation unit #includes the reference's src/loop.c so that its
 * static tick phases -- trace() loop.c:375, deposit() loop.c:388,
 * merge_pars() loop.c:610 and update_pars() loop.c:647 -- and its ray array
 * r[] become callable. It is linked with the reference's raytrace.c,
 * pluecker-sse.c, sph-depth.c, solve.c, tabfun.c, atomic-rate.c, units.c and
 * support/lsoda, all compiled from the reference tree with the reference's
 * flags (see oracle/Makefile). The globals that the reference's config.c and
 * psystem.c would own are defined here and filled from the caller's arrays,
 * mirroring psystem_read_epoch() psystem.c:300-379 and cfg_init()
 * config.c:60-167 for the fields the hot path reads.
 *
 * What it bypasses: emit_rays() (loop.c:163) -- rays come from the caller --
 * and all IO (config parsing, snapshot reading, output writing). Functions on
 * those paths are stubs that abort if reached.
 *
 * Test infrastructure only: the product never links or calls this. */
#include "loop.c"

/* ---- globals normally owned by config.c / psystem.c / stat.c / epochs.c --- */
config_t CFG[1];
gsl_rng *RNG = NULL;
int CFG_WRITE_INIT = 0;
int CFG_ISOTHERMAL = 1;
int CFG_ADIABATIC = 0;
int CFG_ON_THE_SPOT = 1;
int CFG_COMOVING = 0;
int CFG_DUMP_HOTSPOTS = 0;
int CFG_H_ONLY = 1;
int CFG_TRACE_ONLY = 0;
int CFG_NO_PHOTON = 0;
int CFG_SECONDARY_IONIZATION = 0;
int CFG_OCTTREE_PPC = 8;
int CFG_DISABLE_LTE = 1;
int CFG_PRINT_RAYS = 0;
int CFG_ENABLE_EOS = 0;
double CFG_EOS_CLOUD_TEMPERATURE = 1e3;
double CFG_RECOMBINE_THRESHOLD = 0.1;
double CFG_BOOST_SOURCE_FACTOR = 1.0;
double CFG_FAKE_TEMPERATURE = -1;
double C_1_CMH = 3.0835455558318480e+21;
double C_1_GRAMH = 1.9847005219450705e+43;
double C_1_SECH = 3.08568025e+16;
double C_OMEGA_L = 0.74;
double C_OMEGA_M = 0.26;
double C_OMEGA_B = 0.044;
double C_H = 0.72;
double C_HMF = 0.76;
double C_HEMF = 0.24;
Epoch *EPOCHS = NULL;
/* lte.c is built in ref_lte.c; secion.c is linked from the reference. */
int N_EPOCHS = 0;
PSystem psys = {0};
stat_t stat = {0};

extern double units_init();
extern void ar_init(const char *filename);
extern void xs_init(const char *filename);
extern void rt_switch_epoch(int i);
extern int step_evolve(void *control, Step *step);

static Epoch harness_epoch;
static int tree_built = 0;

/* ---- stubs for functions that are only on bypassed paths ---------------- */
static void bypassed(const char *what) {
	fprintf(stderr, "oracle harness: %s is outside the compared path\n", what);
	abort();
}
void psystem_stat(const char *c) { (void)c; bypassed("psystem_stat"); }
void stat_write(int n) { (void)n; bypassed("stat_write"); }
void stat_reset() { bypassed("stat_reset"); }
void stat_stop() { bypassed("stat_stop"); }
void psystem_write_output(int n) { (void)n; bypassed("psystem_write_output"); }
/* (psystem_weight_srcs() is the reference's own, sources.c built in
 * ref_sources.c; the source rays' energy is not compared: one fixed energy) */
static double harness_spec_freq = 0.0;
double spec_gen_freq(const int id) {
	(void)id;
	if (!(harness_spec_freq > 0.0)) bypassed("spec_gen_freq");
	return harness_spec_freq;
}
int spec_get(const char *name) { (void)name; bypassed("spec_get"); return 0; }
double spec_N_from_lum(const int id, double lum) { (void)id; (void)lum; bypassed("spec_N_from_lum"); return 0; }
double eos_get_cloud_fraction(const double d) { (void)d; bypassed("eos_get_cloud_fraction"); return 0; }
double eos_get_egyhot(const double d) { (void)d; bypassed("eos_get_egyhot"); return 0; }

/* ---- exported API (ctypes) ---------------------------------------------- */
typedef struct {
	float s[3];
	float dir[3];
	double Nph;
	double freq;
	double length;
} ref_ray;

int ref_setup(const char *rates_path, double h, double hmf,
		double len_cmh, double mass_gramh, double time_sh,
		int isothermal, int on_the_spot, int h_only, int adiabatic) {
	C_H = h;
	C_HMF = hmf;
	C_HEMF = 1.0 - hmf;
	C_1_CMH = len_cmh;
	C_1_GRAMH = mass_gramh;
	C_1_SECH = time_sh;
	CFG_ISOTHERMAL = isothermal;
	CFG_ON_THE_SPOT = on_the_spot;
	CFG_H_ONLY = h_only;
	CFG_ADIABATIC = adiabatic;
	CFG_SECONDARY_IONIZATION = 0;
	units_init();
	ar_init(rates_path);
	xs_init(NULL);
	return 0;
}

void ref_set_threads(int n) { omp_set_num_threads(n); }
int ref_max_threads(void) { return omp_get_max_threads(); }

/* Unit constants the product must reproduce (units.c:24-62). */
void ref_units(double out[16]) {
	out[0] = U_CM; out[1] = U_GRAM; out[2] = U_SEC; out[3] = U_MYR;
	out[4] = U_EV; out[5] = U_MPROTON; out[6] = C_BOLTZMANN;
	out[7] = C_H_PER_MASS; out[8] = C_HE_PER_MASS; out[9] = C_HI_ENERGY;
	out[10] = U_MPROTON_OVER_C_BOLTZMANN; out[11] = C_BOLTZMANN_OVER_U_MPROTON;
	out[12] = U_ERG; out[13] = U_KPC; out[14] = C_HEI_ENERGY; out[15] = C_HEII_ENERGY;
}

double ref_sph_depth(double r_h) { return sph_depth(r_h); }
double ref_ar_get(int id, double logT) { return ar_get(id, logT); }
double ref_xs_get(int id, double freq) { return xs_get(id, freq); }
/* Column ids in the order: HIci HIIrcA HIIrcB HIIrccA HIIrccB HIcic HIcec Brem
 * Compton XS_HI XS_HeI XS_HeII. */
void ref_ids(int out[12]) {
	out[0] = AR_HI_CI; out[1] = AR_HII_RC_A; out[2] = AR_HII_RC_B;
	out[3] = AR_HII_RCC_A; out[4] = AR_HII_RCC_B; out[5] = AR_HI_CIC;
	out[6] = AR_HI_CEC; out[7] = AR_E_BREMC; out[8] = AR_E_COMPC;
	out[9] = XS_HI; out[10] = XS_HEI; out[11] = XS_HEII;
}

/* Fill psys the way psystem_read_epoch() (psystem.c:300-379) does for the
 * fields the hot path reads; flag may be NULL. */
int ref_load_particles(size_t n, const float *pos, const float *mass,
		const float *sml, const float *rho, const float *ie,
		const float *xHI, const float *ye, const int8_t *flag, double boxsize) {
	psys.npar = n;
	psys.npar_max = n;
	psys.boxsize = boxsize;
	psys.pos = calloc(n, sizeof(float) * 3);
	psys.mass = calloc(n, sizeof(float));
	psys.sml = calloc(n, sizeof(float));
	psys.rho = calloc(n, sizeof(float));
	psys.ie = calloc(n, sizeof(float));
	psys.yeMET = calloc(n, sizeof(float));
	psys.lambdaH = calloc(n, sizeof(double));
	psys.lambdaHeI = calloc(n, sizeof(double));
	psys.lambdaHeII = calloc(n, sizeof(double));
	for (int i = 0; i < 3; i++) {
		psys.yGrec[i] = calloc(n, sizeof(float));
		psys.yGdep[i] = calloc(n, sizeof(float));
	}
	psys.heat = calloc(n, sizeof(float));
	psys.lasthit = calloc(n, sizeof(intptr_t));
	psys.hits = calloc(n, sizeof(int));
	psys.flag = calloc(n, sizeof(int8_t));
	psys.id = calloc(n, sizeof(uint64_t));
	memcpy(psys.pos, pos, sizeof(float) * 3 * n);
	memcpy(psys.mass, mass, sizeof(float) * n);
	memcpy(psys.sml, sml, sizeof(float) * n);
	memcpy(psys.rho, rho, sizeof(float) * n);
	memcpy(psys.ie, ie, sizeof(float) * n);
	memcpy(psys.yeMET, ye, sizeof(float) * n);
	if (flag) memcpy(psys.flag, flag, n);
	for (size_t i = 0; i < n; i++) {
		const double xHII = 1.0 - xHI[i];
		psys_set_lambdaH(i, xHI[i], xHII);
		double yeMET = fdim(psys.yeMET[i], xHII);
		if (!CFG_H_ONLY) {      /* psystem.c:350-357 */
			double xHeII = yeMET * C_HMF / (1 - C_HMF) * 4;
			double xHeIII = fdim(xHeII, 1.0);
			xHeII = fmin(1.0, xHeII);
			xHeIII = fmin(1.0 - xHeII, xHeIII);
			psys_set_lambdaHe(i, 1.0 - xHeII - xHeIII, xHeII, xHeIII);
			yeMET = fdim(yeMET, (xHeII + 2 * xHeIII) * (1 - C_HMF) / C_HMF * 0.25);
		}
		psys.yeMET[i] = yeMET;
		psys.id[i] = i;
	}
	psys.tick = 0;
	active = bitmask_alloc(n);     /* as run_epoch() loop.c:89-90 */
	bitmask_clear_all(active);
	harness_epoch.nray = 0;
	psys.epoch = &harness_epoch;
	return 0;
}

/* rt_switch_epoch(0) sizes its pool and next[] from the loaded particle
 * count, so every build here takes that path (the arrays of an earlier
 * build are simply dropped). */
int ref_build_tree(int ppc) {
	CFG_OCTTREE_PPC = ppc;
	rt_switch_epoch(0);
	tree_built = 1;
	return 0;
}

size_t ref_rt_trace(const float s[3], const float dir[3], float dist,
		Xtype **x, size_t *size) {
	return rt_trace(s, dir, dist, x, size);
}
void ref_free(void *p) { free(p); }

int ref_set_rays(size_t n, const ref_ray *rays, long tick, double tick_time) {
	ARRAY_RESIZE(r, struct r_t, n);
	for (size_t i = 0; i < n; i++) {
		for (int d = 0; d < 3; d++) {
			r[i].s[d] = rays[i].s[d];
			r[i].dir[d] = rays[i].dir[d];
		}
		r[i].Nph = rays[i].Nph;
		r[i].freq = rays[i].freq;
		r[i].length = rays[i].length;
		r[i].type = -1;
		r[i].isrc = 0;
	}
	r_length = n;
	harness_epoch.nray = n;
	psys.tick = tick;
	psys.tick_time = tick_time;
	return 0;
}

/* The tick phases of run_epoch() loop.c:131-147, one at a time. */
void ref_trace(void) { trace(); }
void ref_deposit(void) { deposit(); }
void ref_merge(void) { merge_pars(); }
void ref_update(void) { update_pars(); }

size_t ref_ray_nhits(size_t i) { return r[i].x_length; }
size_t ref_ray_hits(size_t i, int64_t *ipar, double *d, double *b) {
	for (size_t j = 0; j < r[i].x_length; j++) {
		ipar[j] = r[i].x[j].ipar;
		d[j] = r[i].x[j].d;
		b[j] = r[i].x[j].b;
	}
	return r[i].x_length;
}
size_t ref_active_count(void) { return active_set_length; }
void ref_active(int64_t *out) {
	for (size_t i = 0; i < active_set_length; i++) out[i] = active_set[i];
}

/* Secondary ionisation (psphray.secondaryIonization, secion.c): on/off and
 * its table (secion_init() builds it once). */
extern void secion_init(void);
void ref_set_secondary(int on) {
	static int built = 0;
	CFG_SECONDARY_IONIZATION = on;
	if (on && !built) {
		secion_init();
		built = 1;
	}
}
/* secion_get() for column 0 PhiHI, 1 PhiHeI, 2 Eh. */
double ref_secion_get(int col, double E, double log10x) {
	const int ids[3] = {SECION_PHI_HI, SECION_PHI_HEI, SECION_EH};
	return secion_get(ids[col], E, log10x);
}

/* Helium state (psystem.h:35-36, 49-50) and yeMET. */
void ref_get_he(double *lambdaHeI, double *lambdaHeII, float *yGdepHeI, float *yGdepHeII, float *yeMET) {
	for (size_t i = 0; i < psys.npar; i++) {
		if (lambdaHeI) lambdaHeI[i] = psys.lambdaHeI[i];
		if (lambdaHeII) lambdaHeII[i] = psys.lambdaHeII[i];
		if (yGdepHeI) yGdepHeI[i] = psys.yGdepHeI[i];
		if (yGdepHeII) yGdepHeII[i] = psys.yGdepHeII[i];
		if (yeMET) yeMET[i] = psys.yeMET[i];
	}
}
void ref_set_he(const double *lambdaHeI, const double *lambdaHeII) {
	for (size_t i = 0; i < psys.npar; i++) {
		if (lambdaHeI) psys.lambdaHeI[i] = lambdaHeI[i];
		if (lambdaHeII) psys.lambdaHeII[i] = lambdaHeII[i];
	}
}

/* yGrecHII (psystem.h:56): the recombination photons of runs not on the
 * spot, which update_pars() carries through step_evolve() (loop.c:680,756). */
void ref_get_ygrec(float *out) {
	for (size_t i = 0; i < psys.npar; i++) out[i] = psys.yGrecHII[i];
}
void ref_set_ygrec(const float *in) {
	for (size_t i = 0; i < psys.npar; i++) psys.yGrecHII[i] = in[i];
}
/* all three species' recombination photons (psystem.h:56-58) */
void ref_get_ygrec3(float *a, float *b, float *c) {
	for (size_t i = 0; i < psys.npar; i++) {
		a[i] = psys.yGrec[0][i];
		b[i] = psys.yGrec[1][i];
		c[i] = psys.yGrec[2][i];
	}
}
void ref_set_ygrec3(const float *a, const float *b, const float *c) {
	for (size_t i = 0; i < psys.npar; i++) {
		psys.yGrec[0][i] = a[i];
		psys.yGrec[1][i] = b[i];
		psys.yGrec[2][i] = c[i];
	}
}

void ref_get_state(double *lambdaH, float *ie, float *yGdepHI, float *heat,
		int32_t *hits, int64_t *lasthit) {
	for (size_t i = 0; i < psys.npar; i++) {
		if (lambdaH) lambdaH[i] = psys.lambdaH[i];
		if (ie) ie[i] = psys.ie[i];
		if (yGdepHI) yGdepHI[i] = psys.yGdepHI[i];
		if (heat) heat[i] = psys.heat[i];
		if (hits) hits[i] = psys.hits[i];
		if (lasthit) lasthit[i] = psys.lasthit[i];
	}
}
void ref_set_state(const double *lambdaH, const float *ie, const int64_t *lasthit) {
	for (size_t i = 0; i < psys.npar; i++) {
		if (lambdaH) psys.lambdaH[i] = lambdaH[i];
		if (ie) psys.ie[i] = ie[i];
		if (lasthit) psys.lasthit[i] = lasthit[i];
	}
}

/* stat counters and per-phase timers (stat.h:37-60) */
void ref_stats(double out[8]) {
	out[0] = (double)stat.total_deposit_count;
	out[1] = (double)stat.saturated_deposit_count;
	out[2] = stat.raytrace_time;
	out[3] = stat.deposit_time;
	out[4] = stat.merge_time;
	out[5] = stat.update_time;
	out[6] = (double)stat.evolve_count;
	out[7] = stat.lost_photon_count_sum;
}
void ref_reset_stats(void) { memset(&stat, 0, sizeof(stat)); }

/* One call of step_evolve() solve.c:317 per Step, for solver parity. */
int ref_step_evolve(Step *steps, size_t n) {
	void *control = step_evolve_prepare();
	for (size_t i = 0; i < n; i++) step_evolve(control, &steps[i]);
	step_evolve_free(control);
	return 0;
}
size_t ref_sizeof_step(void) { return sizeof(Step); }

/* ---- source rays: emit_rays() loop.c:163-373, on the spot ---------------- */
/* Point sources with luminosity histories (psystem.h:7-25): source i has
 * nhist[i] entries of (hist_ticks, hist_ngd) from offset hist_off[i]. */
void ref_set_sources(int n, const double *pos, const int64_t *hist_ticks, const double *hist_ngd,
		const int *hist_off, const int *nhist, const int64_t *lastemit) {
	psys.srcs = calloc((size_t)n, sizeof(Source));
	psys.nsrcs = (size_t)n;
	for (int i = 0; i < n; i++) {
		Source *S = &psys.srcs[i];
		for (int d = 0; d < 3; d++) S->pos[d] = pos[3 * i + d];
		S->type = PSYS_SRC_POINT;
		S->specid = 0;
		S->lastemit = (intptr_t)lastemit[i];
		S->ticks = malloc(sizeof(intptr_t) * (size_t)nhist[i]);
		S->Ngamma_dots = malloc(sizeof(double) * (size_t)nhist[i]);
		for (int k = 0; k < nhist[i]; k++) {
			S->ticks[k] = (intptr_t)hist_ticks[hist_off[i] + k];
			S->Ngamma_dots[k] = hist_ngd[hist_off[i] + k];
		}
		S->ticks_length = S->ticks_size = (size_t)nhist[i];
		S->Ngamma_dots_length = S->Ngamma_dots_size = (size_t)nhist[i];
		S->cursor = 0;
	}
}

void ref_get_sources(int64_t *lastemit, int64_t *cursor) {
	for (size_t i = 0; i < psys.nsrcs; i++) {
		lastemit[i] = (int64_t)psys.srcs[i].lastemit;
		cursor[i] = (int64_t)psys.srcs[i].cursor;
	}
}

/* One tick of emit_rays() with nray source rays, its source draws made at
 * the uniforms u[0..nray) in draw order (the shim's queue); returns the
 * rays' count and, in the reference's final ray order (sorted by source),
 * each ray's source and photons. The energy is freq for every ray; the
 * directions are not compared. */
int ref_emit_source_rays(int nray, int64_t tick, double tick_time, double freq, const double *u, int64_t *isrc,
		double *nph) {
	const int saved = CFG_ON_THE_SPOT;
	CFG_ON_THE_SPOT = 1;
	psys.tick = (intptr_t)tick;
	psys.tick_time = tick_time;
	harness_epoch.nray = (size_t)nray;
	harness_spec_freq = freq;
	oracle_shim_queue_uniforms(u, (size_t)nray);
	emit_rays();
	oracle_shim_queue_uniforms(NULL, 0);
	harness_spec_freq = 0.0;
	CFG_ON_THE_SPOT = saved;
	for (size_t i = 0; i < r_length; i++) {
		isrc[i] = (int64_t)r[i].isrc;
		nph[i] = r[i].Nph;
	}
	return (int)r_length;
}
