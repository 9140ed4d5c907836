/* psg.h -- C ABI of the B200 trace -> deposit -> solve library (libpsg.so).
 *
 * Drop-in for the hot path of psphray (rainwoodman/psphray). Each entry
 * point names the reference function it replaces. Conventions:
 *   - every call returns PSG_OK (0) or a negative PSG_E_* code; nothing traps
 *     (the reference raises SIGTRAP through ERROR(), support/messages.h:17);
 *     psg_last_error() gives the message of the last failure of a context;
 *   - host buffers belong to the caller, device buffers to the library;
 *   - one host thread per context; calls on one context are serialised on the
 *     context's own CUDA stream;
 *   - particles keep the caller's order: particle index ipar is the position
 *     in the arrays given to psg_load_particles().
 */
#ifndef PSG_H
#define PSG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PSG_OK 0
#define PSG_E_INVAL (-1)     /* bad argument or call order */
#define PSG_E_CUDA (-2)      /* CUDA runtime error */
#define PSG_E_NOMEM (-3)     /* device or host allocation failed */
#define PSG_E_OVERFLOW (-4)  /* a fixed capacity was exceeded (tree depth, table size) */
#define PSG_E_IO (-5)        /* file missing or malformed */
#define PSG_E_DEVICE (-6)    /* a kernel raised its status word (NaN, solver failure) */

/* ---- units: units_init() src/units.c:66-104, defaults src/config.c:15-23 -- */
typedef struct {
	double h;            /* cosmology.h */
	double hmf;          /* cosmology.hmf, hydrogen mass fraction */
	double length_cmh;   /* units.lengthCMh */
	double mass_gramh;   /* units.massGramh */
	double time_sh;      /* units.timeSh */
} psg_unit_params;

typedef struct {
	double CM, GRAM, SEC, M, KM, KPC, YR, MYR, KG, MSUN, MPROTON, KELVIN;
	double BOLTZMANN, J, EV, ERG, RY_ENG;
	double H_PER_MASS, HE_PER_MASS, HI_ENERGY, HEI_ENERGY, HEII_ENERGY;
	double MPROTON_OVER_BOLTZMANN, BOLTZMANN_OVER_MPROTON;
	double hmf, hemf;
} psg_units;

/* Fills *u from *p. Replaces units_init() units.c:66. */
int psg_units_init(const psg_unit_params *p, psg_units *u);

/* ---- atomic-rate table: tabfun_init() src/tabfun.c:60-130 + ar_init()
 * src/atomic-rate.c:66-87. Columns, after unit scaling: */
enum {
	PSG_AR_HI_CI = 0, PSG_AR_HII_RC_A, PSG_AR_HII_RC_B, PSG_AR_HII_RCC_A, PSG_AR_HII_RCC_B,
	PSG_AR_HI_CIC, PSG_AR_HI_CEC, PSG_AR_E_BREMC, PSG_AR_E_COMPC,
	PSG_AR_HEI_CI, PSG_AR_HEII_CI, PSG_AR_HEII_RC_A, PSG_AR_HEII_RC_B, PSG_AR_HEIII_RC_A,
	PSG_AR_HEIII_RC_B, PSG_AR_NCOLS
};
typedef struct {
	int nrows;
	double min, max, step, step_inv;
	double *logT;                 /* first column of the file, nrows */
	double *col[PSG_AR_NCOLS];    /* scaled to internal units, nrows each */
} psg_rate_table;

/* Parses the 14-character fixed-width table at path. Replaces ar_init(). */
int psg_rate_table_load(const char *path, const psg_units *u, psg_rate_table *t);
void psg_rate_table_free(psg_rate_table *t);
/* ar_get() atomic-rate.c:89 / tabfun_get() tabfun.c:38-58. */
double psg_ar_get(const psg_rate_table *t, int col, double logT);

/* ---- cross sections: xs_init(NULL) atomic-rate.c:93-124 with the analytic
 * fits of src/verner.F90, 16384 rows over 1-100 Ry. */
enum { PSG_XS_HI = 0, PSG_XS_HEI, PSG_XS_HEII, PSG_XS_NSPECIES };
typedef struct {
	int nrows;
	double min, max, step, step_inv;
	double *eng;
	double *sigma[PSG_XS_NSPECIES];
	double cut[PSG_XS_NSPECIES];
} psg_xs_table;
int psg_xs_table_build(const psg_units *u, psg_xs_table *t);
void psg_xs_table_free(psg_xs_table *t);
/* xs_get() atomic-rate.c:126-131. */
double psg_xs_get(const psg_xs_table *t, int species, double freq);

/* ---- SPH column-depth table (src/kernel.akline format: one double per line,
 * trailing comma). *n receives the count (4096 for the reference table). */
int psg_kernel_table_load(const char *path, double *out, int cap, int *n);
/* sph_depth() src/sph-depth.c:26-33. */
double psg_sph_depth(const double *table, int n, double r_h);

/* ---- context -------------------------------------------------------------- */
typedef struct psg_context psg_context;

int psg_create(psg_context **ctx, int device);
void psg_destroy(psg_context *ctx);
const char *psg_last_error(const psg_context *ctx);
/* With on != 0, psg_run_ticks*() bracket every kernel launch with CUDA
 * events on the context's stream and report per-kernel device time. */
int psg_set_timing(psg_context *ctx, int on);
/* Run the context's work on the caller's CUDA stream (a cudaStream_t passed
 * as void*; NULL restores the context's own stream). No reference
 * counterpart: the reference has no device. */
int psg_set_stream(psg_context *ctx, void *stream);
/* The SASS and PTX architecture versions (major*10 + minor, 100 for
 * sm_100a) of the library's device code as loaded on the context's device
 * (cudaFuncGetAttributes). No reference counterpart: a build check. */
int psg_device_arch(psg_context *ctx, int *binary_version, int *ptx_version);

/* Physics switches, the config.c flags that the path reads. */
typedef struct {
	int isothermal;          /* psphray.isothermal */
	int on_the_spot;         /* psphray.onTheSpot; 0: case-A recombination, the photons
	                            collected in yGrecHII and re-emitted as recombination
	                            rays (psg_set_recombination) */
	int h_only;              /* psphray.HOnly; 0: helium as well (HeI, HeII, HeIII) */
	int adiabatic;           /* psphray.adiabatic */
	int euler;               /* step_evolve_euler() solve.c:225-316 (a build without
	                            USE_LSODA) instead of the adaptive integrator */
	int secondary_ionization;   /* psphray.secondaryIonization: the deposit's
	                            secondary ionisation and heating (loop.c:513-552) */
} psg_flags;

/* secion_init() secion.c:74-98: the secondary-ionisation fractions of
 * Ricotti, Gnedin & Shull (2002, ApJ 575, 33) -- PhiHI, PhiHeI and the
 * heating fraction Eh -- tabulated on PSG_SECION_NE energies above
 * threshold (10 to 200 eV) by PSG_SECION_NX values of log10 x_e (-8 to 0):
 * out[3][PSG_SECION_NE][PSG_SECION_NX]. Used by psg_set_physics with
 * secondary_ionization; exposed for tests. */
#define PSG_SECION_NE 4096
#define PSG_SECION_NX 1024
int psg_secion_table_build(const psg_units *u, double *out);

/* Upload units, tables and flags. Must precede psg_load_particles() (the
 * ye block is split into hydrogen, helium and metal electrons at load with
 * the HOnly flag set then). */
int psg_set_physics(psg_context *ctx, const psg_units *u, const psg_rate_table *ar,
		const psg_xs_table *xs, const double *kernel, int kernel_n, const psg_flags *flags);

/* Particle arrays (reference storage types, psystem.h:32-78). xHI and ye are
 * the snapshot blocks; lambdaH and yeMET are derived as psystem_read_epoch()
 * psystem.c:340-356 does. flag may be NULL (bit 0 = PF_INVALID). */
typedef struct {
	size_t n;
	const float *pos;    /* [n][3] */
	const float *mass, *sml, *rho, *ie, *xHI, *ye;
	const int8_t *flag;
	double boxsize;
} psg_particles;
int psg_load_particles(psg_context *ctx, const psg_particles *p);

/* Octree over [0, boxsize)^3 with at most ppc particles per leaf, built on
 * the device. Replaces rt_switch_epoch() raytrace.c:41-151 (same cells, same
 * leaf boxes). */
int psg_build_tree(psg_context *ctx, int ppc);

typedef struct {
	size_t ncells, nleaves, skipped;
	int depth;
} psg_tree_info;
int psg_get_tree_info(psg_context *ctx, psg_tree_info *info);
/* Cells in depth-first order (children 0..7): boxes, the index just past each
 * cell's subtree, and the first particle (in leaf order) of each cell; and
 * the leaf-order particle permutation. Arrays sized from psg_get_tree_info;
 * pstart has ncells+1 entries. Any pointer may be NULL. */
int psg_get_tree(psg_context *ctx, float *bot, float *top, int32_t *skip, int32_t *pstart,
		int32_t *order);

/* ---- rays and hits --------------------------------------------------------- */
typedef struct {
	float s[3];
	float dir[3];
	double Nph;
	double freq;
	double length;
} psg_ray;                  /* struct r_t loop.c:21-35 without the bookkeeping */

typedef struct {
	int64_t ipar;
	double d;
	double b;
} psg_xtype;                /* Xtype psystem.h:108-112 */

/* One ray, rt_trace() raytrace.c:153 signature plus the context: hits sorted
 * by (d, ipar) -- the reference's trace() order (loop.c:383) with ties made
 * deterministic. *x is (re)allocated with malloc as in the reference (caller
 * frees); returns the hit count, or (size_t)-1 on error. */
size_t psg_rt_trace(psg_context *ctx, const float s[3], const float dir[3], const float dist,
		psg_xtype **x, size_t *size);

/* Many rays at once, host buffers: offsets[nray+1] and hits in *x (grown with
 * realloc as needed, size in *size). Replaces trace() loop.c:375-386. */
int psg_trace(psg_context *ctx, const psg_ray *rays, size_t nray, int64_t *offsets,
		psg_xtype **x, size_t *size);

/* ---- ticks ----------------------------------------------------------------- */
/* Kernels timed by psg_tick_stats when timing is on (psg_set_timing). */
enum { PSG_K_TRACE_COUNT = 0, PSG_K_TRACE_FILL, PSG_K_SORT, PSG_K_SLOTS, PSG_K_DEPOSIT,
	PSG_K_UPDATE, PSG_K_EMIT, PSG_K_NKERNELS };
typedef struct {
	double hits;            /* sum of hit-list lengths, stat.total_deposit_count */
	double saturated;       /* deposits capped at the neutral atoms, loop.c:482-485 */
	double active;          /* particle updates, stat.evolve_count */
	double lost_photons;    /* photons left in rays at their end */
	double trace_ms, tick_ms;   /* device time: trace+sort+slots, then the tick loop */
	double launches;        /* kernels of this library launched by the call */
	double kernel_ms[PSG_K_NKERNELS];        /* per kernel group, with timing on */
	double kernel_launches[PSG_K_NKERNELS];
	double surrogate_accepted;  /* particle updates taken from the surrogate (psg_set_surrogate) */
	double rec_rays;        /* recombination rays emitted (stat.rec_ray_count) */
	double rec_photons;     /* photons they carried (stat.rec_photon_count) */
	double host_syncs;      /* times the call waited for the device (host reads of device counts) */
} psg_tick_stats;

/* Runs nticks ticks; rays holds nray_per_tick rays for each tick, tick by
 * tick (host buffer). Tick k (0-based) is the reference's psys.tick =
 * first_tick + k. Per tick: trace, deposit, merge, update -- run_epoch()
 * loop.c:128-147 without the source half of emit_rays(). Not on the spot,
 * each tick also emits its recombination rays on the device first (see
 * psg_set_recombination) and the ticks run one at a time. stats may be
 * NULL. */
int psg_run_ticks(psg_context *ctx, const psg_ray *rays, size_t nray_per_tick, size_t nticks,
		int64_t first_tick, double tick_time, psg_tick_stats *stats);
/* Same with rays already in device memory. */
int psg_run_ticks_device(psg_context *ctx, const psg_ray *d_rays, size_t nray_per_tick,
		size_t nticks, int64_t first_tick, double tick_time, psg_tick_stats *stats);

/* ---- launch shapes and their autotuner ------------------------------------ */
/* No reference counterpart (the reference has one CPU code path): the shapes
 * of the device path that do not change its results beyond FP64 rounding,
 * chosen per device by timing. */
typedef struct {
	int trace_warps;        /* warps per traversal block, 1-16 (default 4) */
	int deposit_long;       /* rays with more hits than this take a 128-thread group (default 96) ... */
	int deposit_mid;        /* ... more than this a 512-thread block (default 384); fewer take a warp */
	int update_minblocks;   /* 3 or 4: the integrator's registers capped for that many resident
	                         * blocks per multiprocessor (spilling the rest); 1: uncapped (default) */
	int leaf_size;          /* particles per octree leaf: the reference's CFG_OCTTREE_PPC, 8; the hit
	                         * lists are bit-exact only with the reference's leaves, so it is reported,
	                         * never searched */
	int run_short;          /* a particle's deposits of one tick up to this many (4, 8 or 16; default
	                         * 16) are put in hit order where they are summed; longer runs are sorted
	                         * first. The sums are the same either way. */
	int update_order;       /* 1 (default): the integrator claims first the particles that look slow
	                         * (no carried step proposal, a proposal under a quarter of the step, or
	                         * more photons absorbed than neutral atoms), then the rest; 0: in particle
	                         * order. Which lane integrates a particle changes, its result does not. */
} psg_tune;
int psg_set_tune(psg_context *ctx, const psg_tune *tune);
int psg_get_tune(psg_context *ctx, psg_tune *tune);
/* Times candidate shapes on one batch of the caller's device rays (R rays
 * per tick, K ticks, as psg_run_ticks_device), each `reps` times, one
 * dimension after another (traversal warps, deposit thresholds, integrator
 * registers, short-run threshold, integrator order), and keeps the fastest. The particle state is restored after
 * every trial, so the call does not advance the run. The result becomes the
 * context's shapes and the device's cached shapes, which contexts created
 * later on that device start from. *best_ms: the kept shape's batch time. */
int psg_autotune(psg_context *ctx, const psg_ray *d_rays, size_t R, size_t K, int64_t first_tick,
		double tick_time, int reps, psg_tune *out, double *best_ms);

/* ---- recombination rays (psphray.onTheSpot = false) ---------------------- */
/* The recombination half of emit_rays() loop.c:197-232, 273-300, 322-368:
 * from the second tick on, the particles hit in the previous tick by its
 * source rays (and by its first recombination ray, merge_pars()
 * loop.c:628-630) emit nrec rays per tick and species (HII; with helium also
 * HeII and HeIII), each drawing its particle with weight yGrec/xHI; a ray
 * starts at the particle, goes in an isotropic direction for 0.2 box
 * sides, carries the particle's yGrec times NH (HII) or NHe split evenly
 * over the rays that drew it, and has an energy drawn from lte_gen_freq()
 * lte.c:36-44 at the particle's temperature (or the species' edge with
 * disable_lte, psphray.disableLTE). The photons leave yGrec. With
 * nrec < 0 every such particle with yGrecHII > threshold
 * (psphray.recombineThreshold) emits one ray; with nrec = 0 none is emitted
 * and the photons stay in yGrecHII. Defaults: nrec 100 (epoch
 * nrec, epochs.c:29), threshold 0.1, LTE on, seed 0. The draws are this
 * library's own stream (Philox4x32-10, streams 4-6). */
int psg_set_recombination(psg_context *ctx, int nrec, double threshold, int disable_lte, uint64_t seed);
/* The recombination rays of the last tick run, in the order they were
 * traced (by species, then emitting particle), with each emitter's caller
 * index and the ray's type (0 HII, 1 HeII, 2 HeIII recombination, as r_t's
 * type, loop.c:264-266); *n receives their number (rays, ipar and type may
 * be NULL). */
int psg_get_rec_rays(psg_context *ctx, psg_ray *rays, int64_t *ipar, int32_t *type, size_t cap, size_t *n);
/* yGrecHII (psystem.h:56) and the tick each particle was last hit by a
 * source ray (-1: never; the next tick's emitters are those of the
 * previous tick), caller order. Any pointer may be NULL. */
int psg_get_rec_state(psg_context *ctx, float *yGrecHII, int32_t *srcmark);
int psg_set_rec_state(psg_context *ctx, const float *yGrecHII, const int32_t *srcmark);

/* ---- sources and ray emission on the device -------------------------------- */
/* Source rays of emit_rays() loop.c:163-373. A source is psystem.h's Source: position, type, spectrum and its
 * luminosity history (Ngamma_dot from ticks[k] on, sources.c:58-66). */
#define PSG_SRC_PLANE 0     /* PSYS_SRC_PLANE psystem.h:4 */
#define PSG_SRC_POINT 1     /* PSYS_SRC_POINT psystem.h:5 */
typedef struct {
	int type;               /* PSG_SRC_POINT or PSG_SRC_PLANE */
	int specid;             /* index into the spectra of psg_set_sources */
	double pos[3];
	double dir[3];          /* plane sources: the direction of every ray */
	double a[3], b[3];      /* plane sources: unit vectors spanning the plane */
	double radius;          /* plane sources: half side of the emitting square */
	const int64_t *ticks;   /* luminosity history: from tick ticks[k] on, */
	const double *ngamma_dot;   /* photons per unit time ngamma_dot[k] */
	int nhist;              /* entries in the history (>= 1) */
	int64_t lastemit;       /* tick of the last emission (Source.lastemit) */
} psg_source;
typedef struct {
	const double *eng;      /* photon energies (internal units), spectra.c */
	const double *weight;   /* photon-number weight of each energy */
	int n;                  /* 1: monochromatic (spec type 1) */
} psg_spectrum;
#define PSG_MAX_SOURCES 4096

/* Copies the sources, their histories and the spectra to the device and
 * keys the counter-based generator (Philox4x32-10) with seed. Replaces the
 * source and spectrum set-up of psystem_read_source() sources.c and
 * spec_init() spectra.c; the reference's GSL generator has no device
 * counterpart, so the draws are this library's own stream. */
int psg_set_sources(psg_context *ctx, const psg_source *srcs, int nsrc, const psg_spectrum *specs,
		int nspec, uint64_t seed);
/* lastemit and history cursor of every source (after emissions). */
int psg_get_sources(psg_context *ctx, int64_t *lastemit, int32_t *cursor);

/* Emits nray_per_tick source rays for each of nticks ticks into a host
 * buffer (nticks*nray_per_tick rays, tick by tick), advancing the sources'
 * state as the ticks would: per tick, weights = Ngamma_dot*(tick-lastemit)*
 * tick_time (psystem_weight_srcs() sources.c:67-78), a source per ray drawn
 * by weight, the source's photons split evenly over its rays of the tick
 * (loop.c:305-320), isotropic directions for point sources, a uniform point
 * of the square for plane sources, a spectrum energy per ray, length twice
 * the box. */
int psg_emit_rays(psg_context *ctx, size_t nray_per_tick, size_t nticks, int64_t first_tick,
		double tick_time, psg_ray *rays);
/* emit_rays() + the ticks, all on the device (no rays cross the bus). */
int psg_run_ticks_emit(psg_context *ctx, size_t nray_per_tick, size_t nticks, int64_t first_tick,
		double tick_time, psg_tick_stats *stats);

/* Particle state, caller order. Any pointer may be NULL. */
int psg_get_state(psg_context *ctx, double *lambdaH, float *ie, int32_t *hits, int64_t *lasthit);
int psg_set_state(psg_context *ctx, const double *lambdaH, const float *ie, const int64_t *lasthit);
/* Helium state, caller order: lambdaHeI = x_HeI, lambdaHeII = x_HeII
 * (psystem.h:35-36), yeMET (the electrons from metals, after the hydrogen
 * and helium ones are taken out of the ye block at load,
 * psystem.c:340-358) and, not on the spot, the recombination photons per
 * helium atom yGrecHeII, yGrecHeIII (psystem.h:57-58). With HOnly both
 * fractions stay 0 (x_HeIII = 1), as in the reference. Any pointer may be
 * NULL. */
int psg_get_he_state(psg_context *ctx, double *lambdaHeI, double *lambdaHeII, float *yeMET, float *yGrecHeII,
		float *yGrecHeIII);
int psg_set_he_state(psg_context *ctx, const double *lambdaHeI, const double *lambdaHeII, const float *yGrecHeII,
		const float *yGrecHeIII);

/* ---- solver ---------------------------------------------------------------- */
typedef struct {
	double lambdaH, lambdaHeI, lambdaHeII, ie, yeMET, yGdepHI, yGdepHeI, yGdepHeII, heat;
	double time, nH, T, yGrecHII, yGrecHeII, yGrecHeIII, step_remain;
	int refined;
	int64_t ipar;
} psg_step;                 /* Step psystem.h:84-105 */

/* step_evolve() solve.c:317 for n independent steps, on the device; steps
 * are updated in place (host buffer). */
int psg_step_evolve(psg_context *ctx, psg_step *steps, size_t n);

/* psg_step_evolve without any device allocation (no counterpart in the
 * reference): the steps are staged in a fixed buffer inside the library,
 * one per device, of PSG_NOALLOC_MAX_STEPS (16384) steps; larger n is
 * rejected with PSG_E_INVAL. For hosts that cannot allocate device memory
 * while a step is under way: a code whose pool allocator already holds the
 * device's free memory, or one that must avoid the device-wide
 * synchronisation of cudaMalloc/cudaFree. The buffer (2.25 MiB) is reserved
 * when psg_create() runs on the device (it loads the library's module that
 * holds it) and stays until the process exits, so create the context
 * before the host's pool takes the memory. Every call looks the buffer's
 * address up afresh (cheap); a device reset by the host between calls
 * reloads the module on the next call. Calls that overlap in time on one
 * device race on the buffer: serialise them. */
#define PSG_NOALLOC_MAX_STEPS 16384
int psg_step_evolve_noalloc(psg_context *ctx, psg_step *steps, size_t n);

/* ---- snapshots: psystem_write_output() psystem.c:598-690 ------------------ */
/* One psphray-format file (reader-psphray.inc): gas (type 0) and sources
 * (type 5). Array pointers may be NULL: written as zeros, skipped on read. */
typedef struct {
	size_t ngas, nsrc;
	double time;                /* scale factor 1/(1+z) of the output */
	double redshift, boxsize, OmegaM, OmegaL, OmegaB, h;
	float *pos;                 /* [ngas][3] */
	int64_t *id;
	float *mass, *ie, *rho, *ye, *xHI, *sml, *xHeI, *xHeII, *gammaHI;
	int64_t *lasthit;
	int32_t *hits;
	float *src_pos;             /* [nsrc][3] */
	double *ngammas;            /* [nsrc] photons per unit time */
} psg_snapshot;
int psg_snapshot_write(const char *filename, const psg_snapshot *s);
/* counts and constants of a file into s (arrays untouched) */
int psg_snapshot_read_header(const char *filename, psg_snapshot *s);
/* the arrays of a file into the non-NULL pointers of s (s->ngas, s->nsrc
 * must match the file's) */
int psg_snapshot_read(const char *filename, psg_snapshot *s);
/* psystem_write_output(): the particle state on the device, in the caller's
 * order, written with meta's constants, ids and sources (meta->ngas must be
 * the particle count; NULL ids write 0..n-1). xHI = lambdaH, xHeI and xHeII
 * the helium fractions, ye = psys_ye() psystem.h:177 (hydrogen and helium
 * electrons; with HOnly helium counts as fully ionised), gammaHI =
 * yGrecHII (psystem.c:653). */
int psg_write_output(psg_context *ctx, const char *filename, const psg_snapshot *meta);
/* Per-particle deposit counters (psys.hits), caller order; for a resumed run. */
int psg_set_hits(psg_context *ctx, const int32_t *hits);

/* ---- chemistry surrogate: the network and its training ------------------- */
/* No counterpart in the reference (it integrates every particle with LSODA):
 * a 6 -> 64 -> 64 -> 2 perceptron with SiLU activations learns the
 * non-isothermal update of one particle over one step. Parameters are one
 * flat FP32 array: W1[64][8], b1[64], W2[64][64], b2[64], W3[2][64], b3[2]
 * (inputs padded to 8). All pointers are device pointers. */
#define PSG_MLP_NIN 8
#define PSG_MLP_NPARAM 4866
/* y[n][2] = net(x[n][8]) in FP32. */
int psg_mlp_forward(psg_context *ctx, const float *params, const float *x, size_t n, float *y);
/* grad[PSG_MLP_NPARAM + 1]: the gradient of the mean over the n samples of
 * the summed squared error, then the summed squared error itself (also
 * copied to *loss if loss is not NULL). Deterministic. */
int psg_mlp_grad(psg_context *ctx, const float *params, const float *x, const float *t, size_t n,
		float *grad, float *loss);
/* Update log: while set, every non-isothermal tick appends one row of 8
 * floats per particle update to rows (device, cap rows; *count, a device
 * counter the caller zeroes, counts the updates offered): the surrogate's 5
 * inputs (psg_surrogate.cuh: log nH*time, log T, logit lambdaH, log g,
 * log heat/ie), its 2 targets (change of logit lambdaH and of log T) and a
 * zero. rows = NULL switches it off. */
int psg_set_update_log(psg_context *ctx, float *rows, size_t cap, unsigned long long *count);
/* Installs a trained network for the non-isothermal ticks (params as for
 * psg_mlp_forward; x_mu/x_sd[5] normalise the inputs, y_mu/y_sd[2]
 * de-normalise the outputs). Every active particle's step is predicted on
 * the tensor cores (BF16, FP32 accumulation); a prediction whose trapezoid
 * residual exceeds tol (relative, see psg_surrogate.cu) is redone by the
 * integrator. params = NULL switches the surrogate off. */
int psg_set_surrogate(psg_context *ctx, const float *params, const float *x_mu, const float *x_sd,
		const float *y_mu, const float *y_sd, float tol);
/* The installed network on rows of raw inputs (device x[n][8], 5 used):
 * y[n][2] de-normalised outputs, computed exactly as inside the ticks. */
int psg_surrogate_forward(psg_context *ctx, const float *x, size_t n, float *y);
/* One Adam step (step counts from 1). */
int psg_mlp_adam(psg_context *ctx, float *params, const float *grad, float *m, float *v, float lr,
		float beta1, float beta2, float eps, int step);

#ifdef __cplusplus
}
#endif
#endif
