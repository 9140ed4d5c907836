// Internal declarations shared by the libpsg CUDA translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <algorithm>

#include "psg.h"

// Octree keys: 3 bits per level, child k = xbit | ybit<<1 | zbit<<2 as in
// split() raytrace.c:282-287; level 1 in the top bits. 21 levels fit 63 bits.
#define PSG_MAX_LEVELS 21
#define PSG_KEY_OUTSIDE 0xFFFFFFFFFFFFFFFFull
#define PSG_INVALID_BIT 0x80000000u
// Longest hit list sorted in shared memory (16 bytes per hit); longer lists
// take the library segmented sort.
#define PSG_SORT_MAX 8192

// Bits of the device status word.
#define PSG_ST_NAN 1u          // NaN/inf reached a particle state
#define PSG_ST_SOLVER 2u       // the general integrator hit its step limit
#define PSG_ST_IE_NEG 4u       // internal energy would turn negative (solve.c:137-139)
#define PSG_ST_STACK 8u        // traversal stack overflow
#define PSG_ST_SURR 16u        // a surrogate tile's tensor-core step did not complete
#define PSG_ST_SLAB 32u        // a hit list outgrew its slab in a call without host reads (redone)

// scratch slots
enum {
	S_RAYS = 0, S_COUNT, S_OFFSETS, S_RAW_IPAR, S_RAW_D, S_RAW_B, S_KEYS, S_VALS,
	S_HIT_IPAR, S_HIT_KERN, S_ACC, S_ACT, S_CUB, S_TREE, S_MISC, S_REC_U32, S_REC_F64, S_RAYLIST, S_UPD,
	S_EMIT, S_MAP, S_ALONG, S_MLP, S_LOG, S_SURR, S_REC, S_RECW, S_RECK, S_RECRAYS, S_SNAP, S_SCAN, S_SLOTCNT,
	S_SRCHIT,
	S_NSLOTS
};

// Per-call values the tick kernels read on the device, so that a captured
// batch replays unchanged for any first tick and any rays.
struct PsgBatchDev {
	int64_t tick0;          // the batch's first tick (the recombination path advances it per tick)
	double tick_time;       // internal time per tick
	const psg_ray *rays;    // the rays the ticks deposit (the traced ones)
	const psg_ray *src;     // the caller's source rays (recombination path: copied tick by tick)
	int64_t k;              // recombination path: the tick's index within the call
};

struct psg_buf {
	void *p = nullptr;
	size_t bytes = 0;
};

struct psg_context {
	int device = 0;
	cudaStream_t stream = nullptr;       // the stream all work is issued on
	cudaStream_t own_stream = nullptr;   // created with the context
	char err[512] = {0};

	// physics
	int have_physics = 0;
	psg_units u{};
	psg_flags flags{};
	double *d_ar = nullptr;      // [ar_nrows][16]: logT, then the PSG_AR_* columns
	float4 *d_ar_ni = nullptr;   // [ar_nrows][4]: the 7 rates of the non-isothermal
	                             // right-hand side, values then slopes per log T
	double ar_step = 0;
	double ar_ni_scale[8] = {};  // each d_ar_ni column is stored divided by this
	float2 *d_ar_all = nullptr;  // [ar_nrows][16]: (value, slope) of all 15 rate columns (helium)
	double ar_all_scale[PSG_AR_NCOLS] = {};
	int ar_nrows = 0;
	double ar_min = 0, ar_step_inv = 0;
	double *d_xs = nullptr;      // [4][xs_nrows]: energy, sigma_HI, sigma_HeI, sigma_HeII
	int xs_nrows = 0;
	double xs_min = 0, xs_step_inv = 0, xs_cut_HI = 0, xs_cut_HeI = 0, xs_cut_HeII = 0;
	double *d_si = nullptr;      // secondary ionisation: [3][PSG_SECION_NE][PSG_SECION_NX]
	double *d_kernel = nullptr;
	int kernel_n = 0;

	// particles (caller order until the first tree build, leaf order after it)
	size_t n = 0;
	double boxsize = 0;
	float4 *d_psml = nullptr;    // x, y, z, sml
	float *d_mass = nullptr, *d_rho = nullptr, *d_yeMET = nullptr, *d_ie = nullptr;
	int8_t *d_flag = nullptr;
	double *d_lambdaH = nullptr;
	int32_t *d_hits = nullptr;
	int64_t *d_lasthit = nullptr;
	float *d_hstep = nullptr;    // last integrator step proposal, seconds (0: none yet)
	double *d_gcarry = nullptr;  // absorbed photons per H left over by an explicit step
	float *d_ygrec = nullptr;    // yGrecHII: recombination photons per H not yet emitted
	float *d_ygrecHe1 = nullptr, *d_ygrecHe2 = nullptr;  // yGrecHeII, yGrecHeIII (per He)
	double *d_gcarryHe1 = nullptr, *d_gcarryHe2 = nullptr;  // helium photons left by an explicit step
	double *d_lamHeI = nullptr, *d_lamHeII = nullptr;  // x_HeI, x_HeII (with helium or
	                             // secondary ionisation; 0 with HOnly)
	int32_t *d_srcmark = nullptr; // last tick a source ray (or the tick's first recombination
	                             // ray) hit the particle, -1 never: the emitters of the next tick
	uint32_t *d_order = nullptr; // after a tree build the arrays above are in leaf order:
	                             // position k holds the caller's particle d_order[k] (null: caller order)

	// octree, depth-first order
	int have_tree = 0;
	size_t ncell = 0, nleaf = 0, skipped = 0, nvalid = 0;
	int depth = 0;
	float4 *d_cell_lo = nullptr;  // bot.xyz, w = index past the subtree (int bits)
	float4 *d_cell_hi = nullptr;  // top.xyz, w = first particle in leaf order (int bits)
	float4 *d_wide_lo = nullptr;  // level order (siblings contiguous): bot.xyz, w = first child or -1-count
	float4 *d_wide_hi = nullptr;  // top.xyz, w = first particle in leaf order
	float4 *d_leaf_psml = nullptr; // particles in leaf order
	uint32_t *d_leaf_idx = nullptr; // caller index, PSG_INVALID_BIT if flagged

	// sources for device emission: one allocation, layout in psg_emit.cu
	void *d_emit = nullptr;
	int nsrc = 0, nspec = 0, nhist_total = 0, nspec_total = 0;
	uint64_t emit_seed = 0;

	// recombination rays (not on the spot), psg_recomb.cu
	int rec_nrec = 100;          // epoch nrec (epochs.c:29); < 0: every particle above the threshold, 0: none
	double rec_threshold = 0.1;  // psphray.recombineThreshold (config.c:37)
	int rec_disable_lte = 0;     // psphray.disableLTE (config.c:33)
	uint64_t rec_seed = 0;
	double *d_lte = nullptr;     // [3][PSG_LTE_NLOGT][PSG_LTE_NFREQ] cumulative weights
	double lte_freq_min[3] = {}, lte_freq_step[3] = {};
	size_t rec_last = 0;         // recombination rays of the last tick (after the source rays in S_RECRAYS)
	size_t rec_last_R = 0;       // source rays of that tick
	size_t rec_last_kmax = 0;    // capacity of that tick's item arrays (S_RECK)
	int rec_last_threshold = 0;  // that tick ran in threshold mode (its items unsorted, in place)
	size_t src_nray = 0;         // S_SRCHIT: the call's source rays traced and sorted before its ticks ran
	size_t src_nhit = 0;         //   (offsets[src_nray + 1], kernel factor[src_nhit], ipar[src_nhit]; src_nhit
	                             //   a grow-only capacity)

	// chemistry surrogate (not isothermal): weight blob, residual tolerance
	void *d_surr = nullptr;
	float surr_tol = 0.f;
	int surr_on = 0;

	// update log (surrogate training data), caller-owned device buffers
	float *log_buf = nullptr;
	size_t log_cap = 0;
	unsigned long long *log_count = nullptr;

	uint32_t *d_status = nullptr;
	unsigned long long *d_counters = nullptr;   // 32 device counters: 1 capped deposits, 2 lost photons,
	                                            // 3 longest list of a call, 4 longest hit list, 5 hit total,
	                                            // 6 active particles, 7 hits of a call, 8 surrogate accepts,
	                                            // 9 trace ray cursor, 10-13 recombination emission,
	                                            // 14 recombination rays of a call, 15 rays to trace,
	                                            // 16-23 sort size classes, 24 largest tick total of a call
	PsgBatchDev *d_batch = nullptr;             // per-call values read by the tick kernels (device)
	int sms = 148;                              // multiprocessors of the device
	size_t hit_cap = 0;                         // hits the sorted-list buffers hold
	size_t batch_cap = 0;                       // hits the tick batches' per-hit buffers hold
	unsigned sort_grid[8] = {};                 // persistent grids of the per-ray sort's classes
	unsigned trace_grid = 0;                    // persistent grid of the traversal (psg_trace_fill_prepare)
	psg_tune tune{4, 96, 384, 1, 8, 16, 1};        // launch shapes (psg_set_tune, psg_autotune)
	long host_syncs = 0;                        // host synchronisations of the current call
	void *graphs = nullptr;                     // captured tick batches (psg_tick.cu)
	int use_graphs = 1;                         // replay captured batches (0: issue launches one by one)

	// scratch, grown on demand
	psg_buf scratch[S_NSLOTS];
	double sat_frac = 0.0;  // capped share of the last batch's hits (picks the deposit's settle form)
	size_t slab_cap = 0;  // hits each ray can hold in the traversal's output slabs
	int ppc = 8;          // leaf capacity of the current tree
	cudaEvent_t ev[8] = {};
	int timing = 0;
	cudaEvent_t kev[2 * 4096] = {};      // per-launch events when timing is on
	int nkev = 0;
	int kev_kind[4096] = {};
	long launches = 0;                   // kernels of this library launched
};

// error helpers ---------------------------------------------------------------
int psg_fail(psg_context *ctx, int code, const char *fmt, ...);
int psg_cuda_fail(psg_context *ctx, cudaError_t e, const char *what, const char *file, int line);
// Address of psg_step_evolve_noalloc's static buffer on the current device
// (psg_tick.cu); 0 or the cudaError_t of the lookup.
int psg_noalloc_lookup(unsigned char **base);
#define PSG_CUDA(call)                                                               \
	do {                                                                             \
		cudaError_t e_ = (call);                                                     \
		if (e_ != cudaSuccess) return psg_cuda_fail(ctx, e_, #call, __FILE__, __LINE__); \
	} while (0)
#define PSG_CHECK_LAUNCH() PSG_CUDA(cudaGetLastError())

// scratch buffer slot `slot` with at least `bytes`; returns nullptr on failure
void *psg_scratch(psg_context *ctx, int slot, size_t bytes);
// releases the captured tick batches of a context (psg_tick.cu)
void psg_graphs_free(psg_context *ctx);
// copies every per-particle array a tick changes into S_SNAP / back
// (psg_context.cu)
int psg_state_save(psg_context *ctx);
int psg_state_restore(psg_context *ctx);
// the device's cached launch shapes, if psg_autotune ran on it in this process
bool psg_tune_cached(int device, psg_tune *t);
void psg_tune_store(int device, const psg_tune *t);


// Per-launch timing: mark_begin/mark_end bracket a group of launches of one
// kind with events on the context's stream (only when timing is on).
inline void psg_mark_begin(psg_context *ctx, int kind) {
	if (ctx->timing && ctx->nkev < 4096) {
		cudaEventRecord(ctx->kev[2 * ctx->nkev], ctx->stream);
		ctx->kev_kind[ctx->nkev] = kind;
	}
}
inline void psg_mark_end(psg_context *ctx) {
	if (ctx->timing && ctx->nkev < 4096) {
		cudaEventRecord(ctx->kev[2 * ctx->nkev + 1], ctx->stream);
		ctx->nkev++;
	}
}

// permutes every per-particle array by g (new[k] = old[g[k]]) and composes d_order
int psg_permute_particles(psg_context *ctx, const uint32_t *g);

// the surrogate's tick (psg_surrogate.cu)
struct PhysParams;
int psg_surrogate_prepare(psg_context *ctx);
int psg_surrogate_tick(psg_context *ctx, int t, const int32_t *tick_act, const uint32_t *act_ipar,
		const double *act_g, const double *act_heat, const PhysParams &P, const PsgBatchDev *B, uint32_t *rej,
		unsigned *nrej);

// recombination rays (psg_recomb.cu): the tick-by-tick loop used by
// psg_run_ticks_device when not on the spot, and the LTE table build
int psg_run_ticks_rec(psg_context *ctx, const psg_ray *d_rays, size_t R, size_t K, int64_t first_tick,
		double tick_time, psg_tick_stats *stats);
int psg_build_lte(psg_context *ctx, const psg_xs_table *xs);
// the emission of a tick without host reads (its count stays on the
// device), its buffers, and the next tick's emitter marks (psg_recomb.cu)
int psg_rec_prepare(psg_context *ctx);
int psg_rec_emit_enqueue(psg_context *ctx, const PsgBatchDev *B, psg_ray *out, unsigned long long *nlim,
		unsigned long long *recsum);
int psg_rec_mark_enqueue(psg_context *ctx, size_t R, const PsgBatchDev *B);
// the recombination ticks replayed from one captured tick (psg_tick.cu);
// PSG_RETRY: run them one by one instead (first call, slabs too small)
int psg_run_ticks_rec_graph(psg_context *ctx, const psg_ray *d_rays, size_t R, size_t K, int64_t first_tick,
		double tick_time, psg_tick_stats *stats);
#define PSG_RETRY 1
#define PSG_LTE_NLOGT 128
#define PSG_LTE_NFREQ 1024

// tree / trace entry points used across units (psg_trace.cu)
struct PsgTraceFill {
	size_t nhit;                    // hits of all rays
	unsigned long long maxcount;    // longest hit list
	size_t scap;                    // slab capacity per ray
};
int psg_trace_fill(psg_context *ctx, const psg_ray *d_rays, size_t nray, PsgTraceFill *tf);
int psg_trace_sort_prepare(psg_context *ctx, size_t nray, size_t cap, unsigned long long maxcount);
int psg_trace_sort_enqueue(psg_context *ctx, size_t nray, size_t nhit, unsigned long long maxcount, int want_kern,
		size_t r0);
int psg_trace_internal(psg_context *ctx, const psg_ray *d_rays, size_t nray, int want_kern);
int psg_sort_classes(unsigned long long maxcount);
int psg_trace_fill_prepare(psg_context *ctx, size_t nray);
// A recombination tick whose R source rays were traced and sorted with the
// call's (S_SRCHIT): their counts and sorted hits come from there, only the
// emitted rays behind them (at most cap_rec, *nlim of them) are traversed.
int psg_trace_rec_fill_enqueue(psg_context *ctx, const psg_ray *buf, size_t R, size_t cap_rec, const unsigned *nlim,
		size_t cap, const PsgBatchDev *B);
int psg_trace_rec_sort_enqueue(psg_context *ctx, size_t R, size_t nray, unsigned long long maxcount,
		const PsgBatchDev *B);
int psg_trace_src_batch(psg_context *ctx, const psg_ray *d_rays, size_t nray);

// ---- device helpers ------------------------------------------------------------
// Single-rounding float/double ops: the reference is compiled for x86-64 SSE
// without FMA, so each product and sum rounds separately.
__device__ __forceinline__ float rn_fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float rn_fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float rn_fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double rn_dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double rn_dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double rn_dsub(double a, double b) { return __dsub_rn(a, b); }
