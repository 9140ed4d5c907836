// Recombination rays on the device (psphray.onTheSpot = false, hydrogen
// only); replaces the recombination half of emit_rays() loop.c:197-232,
// 273-300, 305-320 and 322-368, with lte_gen_freq() lte.c:36-44 and
// lte_fill() lte.c:46-72.
//
// From the second tick on (loop.c:197), the particles that the previous
// tick's source rays hit -- and those of that tick's first recombination
// ray, which merge_pars() loop.c:628-630 counts in as well -- emit nrec
// rays per species (HII; with helium also HeII and HeIII): each ray draws
// its particle with weight yGrec/xHI (xHI = 0 counts as 1e-10,
// loop.c:207-211), starts at the particle, goes in an isotropic direction
// for a tenth of twice the box (loop.c:169), carries the particle's
// recombination photons yGrec*NH (NHe for helium) split evenly over the
// rays that drew it (loop.c:305-320), and has an energy drawn from the
// species' recombination spectrum sigma(E) E^3 exp(-(E - E_th)/kT) at the
// particle's temperature (lte.c:60-70). The emitted photons leave the
// particle's yGrec (loop.c:345-368). With nrec < 0 every such particle
// above the recombine threshold emits one ray instead (loop.c:221-230; the
// reference reaches that branch through a negative epoch nrec); with nrec
// = 0 none is emitted and the photons stay in yGrecHII (loop.c:180,197).
//
// Emission depends on the previous tick's update, so with recombination
// rays the ticks of a batch run one at a time: emit, then trace, deposit,
// merge and update the tick's source rays and recombination rays together.
//
// Random numbers: psg_philox.cuh, streams 4-8, keyed by the seed of
// psg_set_recombination. The reference draws from GSL's MT19937 and its
// Walker tables (gsl_ran_discrete); the draws here are inverse-CDF draws
// of the same distributions.
#include <math.h>
#include <string.h>

#include <vector>

#include "psg_internal.cuh"
#include "psg_bsort.cuh"
#include "psg_scan.cuh"
#include "psg_helium.cuh"
#include "psg_philox.cuh"
#include "psg_solve.cuh"

int psg_run_ticks_core(psg_context *ctx, const psg_ray *d_rays, size_t R, size_t K, int64_t first_tick,
		double tick_time, psg_tick_stats *stats);

namespace {

inline unsigned nblocks(size_t n, int bs) { return (unsigned)((n + bs - 1) / bs); }

__global__ void k_set_batch_rec(PsgBatchDev *b, int64_t tick, double tick_time, const psg_ray *rays,
		const psg_ray *src, int64_t k) {
	b->tick0 = tick;
	b->tick_time = tick_time;
	b->rays = rays;
	b->src = src;
	b->k = k;
}

__device__ __forceinline__ uint32_t caller_of(const uint32_t *__restrict__ order, uint32_t i) {
	return order ? order[i] : i;
}

// first i in [lo, hi) with cdf[i] >= target, or hi
__device__ __forceinline__ int lower_index(const double *cdf, int lo, int hi, double target) {
	while (lo < hi) {
		const int mid = (lo + hi) >> 1;
		if (cdf[mid] >= target) hi = mid;
		else lo = mid + 1;
	}
	return lo;
}

// The emitters' weights (loop.c:207-211): particles marked in the previous
// tick, yGrecHII / xHI, placed in the caller's particle order (so that the
// draws do not depend on the device's leaf order), and the caller -> leaf
// map.
__global__ void k_rec_weight(size_t n, const PsgBatchDev *__restrict__ B, const int32_t *__restrict__ mark,
		const float *__restrict__ ygrec, const double *__restrict__ lambdaH, const uint32_t *__restrict__ order,
		double *__restrict__ w, uint32_t *__restrict__ leaf_of) {
	const size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
	if (p >= n) return;
	const int32_t prev = (int32_t)(B->tick0 - 1);
	double x = lambdaH[p];
	if (x == 0.0) x = 1e-10;
	const uint32_t c = caller_of(order, (uint32_t)p);
	w[c] = mark[p] == prev ? __ddiv_rn((double)ygrec[p], x) : 0.0;
	leaf_of[c] = (uint32_t)p;
}

// A recombination ray before the sort: key = species << 56 | caller index
// << 24 | draw, val = the emitter (leaf order).
struct RecItem {
	unsigned long long key;
	uint32_t val, spare;
};
struct RecItemLess {
	__device__ __forceinline__ bool operator()(const RecItem &x, const RecItem &y) const { return x.key < y.key; }
};

// nrec draws of species s from the cumulative weights (caller order);
// count[s] = nrec, or 0 when no weight is positive.
__global__ void k_rec_draw(size_t n, int nrec, int s, uint32_t stream, const double *__restrict__ cdf,
		const PsgBatchDev *__restrict__ B, uint64_t seed, const uint32_t *__restrict__ leaf_of,
		RecItem *__restrict__ items, unsigned *__restrict__ count) {
	const int64_t tick = B->tick0;
	const double total = tick > 1 ? cdf[n - 1] : 0.0;       // from the second tick on (loop.c:197)
	const int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k == 0) count[s] = total > 0.0 ? (unsigned)nrec : 0u;
	if (k >= nrec || !(total > 0.0)) return;
	uint32_t x[4];
	draw(x, (uint32_t)k, tick, stream, seed);
	const double target = rn_dmul(u01(x[0], x[1]), total);
	int c = upper_index(cdf, 0, (int)n, target);
	if (c >= (int)n) c = lower_index(cdf, 0, (int)n, total);   // the last particle with weight
	items[k].key = ((unsigned long long)s << 56) | ((unsigned long long)c << 24) | (unsigned long long)k;
	items[k].val = leaf_of[c];
}

// Threshold mode (loop.c:221-230): every marked particle above the
// threshold, flagged in the caller's order (flag[c] for species s at
// s * n + c), and the caller -> leaf map.
__global__ void k_rec_flag(size_t n, const PsgBatchDev *__restrict__ B, const int32_t *__restrict__ mark,
		const float *__restrict__ ygrec, double threshold, const uint32_t *__restrict__ order,
		uint32_t *__restrict__ flag, uint32_t *__restrict__ leaf_of) {
	const size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
	if (p >= n) return;
	const int32_t prev = (int32_t)(B->tick0 - 1);
	const uint32_t c = caller_of(order, (uint32_t)p);
	flag[c] = (B->tick0 > 1 && mark[p] == prev && (double)ygrec[p] > threshold) ? 1u : 0u;
	leaf_of[c] = (uint32_t)p;
}

// The flagged emitters of all species in (species, caller index) order --
// the order the sort gives -- from the scan of the flags; count[s] per
// species.
__global__ void k_rec_place(size_t n, int nspec, const uint32_t *__restrict__ flag,
		const unsigned long long *__restrict__ pos, const uint32_t *__restrict__ leaf_of, RecItem *__restrict__ items,
		unsigned *__restrict__ count) {
	const size_t total = n * (size_t)nspec;
	const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
	if (i == 0)
		for (int s = 0; s < nspec; s++) count[s] = (unsigned)(pos[(size_t)(s + 1) * n] - pos[(size_t)s * n]);
	if (i >= total || !flag[i]) return;
	const size_t s = i / n, c = i - s * n;
	RecItem r;
	r.key = ((unsigned long long)s << 56) | ((unsigned long long)c << 24);
	r.val = leaf_of[c];
	r.spare = 0;
	items[pos[i]] = r;
}

// The LTE tables of the three species (HI, HeI, HeII recombinations).
struct LteView {
	const double *cdf;        // [3][PSG_LTE_NLOGT][PSG_LTE_NFREQ], cumulative weights per row
	double freq_min[3], freq_step[3];
	int disabled;
};

struct RecState {
	float *yg[3];             // yGrecHII, yGrecHeII, yGrecHeIII
};

// Emitter and species of a sorted key; rays of one run share them.
__device__ __forceinline__ unsigned long long run_of(unsigned long long key) { return key >> 24; }

// The rays, in (species, caller index, draw) order -- the reference sorts
// its rays by (type, ipar), loop.c:236. Each ray's photons: the emitter's
// yGrec of the species times NH (HII) or NHe (HeII, HeIII), split over the
// run of rays that drew it (loop.c:277-290, 305-320).
__global__ void k_rec_rays(const unsigned *__restrict__ count, unsigned long long *__restrict__ nlim,
		unsigned long long *__restrict__ recsum, const RecItem *__restrict__ items,
		const PsgBatchDev *__restrict__ B, uint64_t seed,
		const float4 *__restrict__ psml, const float *__restrict__ mass, RecState Y,
		const double *__restrict__ lambdaH, const float *__restrict__ ie, PhysParams P, LteView L, double length,
		psg_ray *__restrict__ out, double *__restrict__ nph_sum) {
	const int M = (int)(count[0] + count[1] + count[2]);
	const int64_t tick = B->tick0;
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i == 0 && nlim) {      // (a captured tick: the traversal's ray limit and the call's ray total)
		*(unsigned *)nlim = (unsigned)M;
		*recsum += (unsigned long long)M;
	}
	if (i >= M) return;
	const uint32_t p = items[i].val;
	const unsigned long long run = run_of(items[i].key);
	const int s = (int)(items[i].key >> 56);
	int c = 1;
	for (int j = i - 1; j >= 0 && run_of(items[j].key) == run; j--) c++;
	for (int j = i + 1; j < M && run_of(items[j].key) == run; j++) c++;
	const double N = rn_dmul((double)mass[p], s == 0 ? P.H_PER_MASS : P.HE_PER_MASS);
	psg_ray r;
	r.Nph = rn_dmul(rn_dmul((double)Y.yg[s][p], N), __ddiv_rn(1.0, (double)c));
	const float4 q = psml[p];
	r.s[0] = q.x;
	r.s[1] = q.y;
	r.s[2] = q.z;
	r.length = length;
	uint32_t x[4];
	draw(x, (uint32_t)i, tick, 5u, seed);
	const double cz = rn_dsub(rn_dmul(2.0, u01(x[0], x[1])), 1.0);
	const double phi = rn_dmul(2.0 * 3.141592653589793, u01(x[2], x[3]));
	const double st = __dsqrt_rn(fmax(0.0, rn_dsub(1.0, rn_dmul(cz, cz))));
	double sp, cp;
	sincos(phi, &sp, &cp);
	r.dir[0] = (float)rn_dmul(st, cp);
	r.dir[1] = (float)rn_dmul(st, sp);
	r.dir[2] = (float)cz;
	if (L.disabled) {
		r.freq = L.freq_min[s];
	} else {
		// psys_T() psystem.h:180-182: T from ie and ye (without yeMET)
		const double T = ieye2T(P, (double)ie[p], ye_he(P, lambdaH[p], P.lamHeI[p], P.lamHeII[p]));
		const double logT = log10(T);
		int row = (int)__ddiv_rn(rn_dsub(logT, 3.0), 7.0 / PSG_LTE_NLOGT);
		if (row < 0) row = 0;
		if (row >= PSG_LTE_NLOGT) row = PSG_LTE_NLOGT - 1;
		const double *cdf = L.cdf + ((size_t)s * PSG_LTE_NLOGT + row) * PSG_LTE_NFREQ;
		draw(x, (uint32_t)i, tick, 6u, seed);
		const double total = cdf[PSG_LTE_NFREQ - 1];
		int j = upper_index(cdf, 0, PSG_LTE_NFREQ, rn_dmul(u01(x[0], x[1]), total));
		if (j >= PSG_LTE_NFREQ) j = lower_index(cdf, 0, PSG_LTE_NFREQ, total);
		r.freq = rn_dadd(L.freq_min[s], rn_dmul(L.freq_step[s], (double)j));
	}
	out[i] = r;
	atomicAdd(nph_sum, r.Nph);
}

// The photons leave the emitter (loop.c:345-368): once per run, ray by ray
// in float as the reference's compound assignment rounds, never below 0.
__global__ void k_rec_purge(const unsigned *__restrict__ count, const RecItem *__restrict__ items,
		const psg_ray *__restrict__ rays, const float *__restrict__ mass, RecState Y, PhysParams P) {
	const int M = (int)(count[0] + count[1] + count[2]);
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= M) return;
	const unsigned long long run = run_of(items[i].key);
	if (i > 0 && run_of(items[i - 1].key) == run) return;
	const uint32_t p = items[i].val;
	const int s = (int)(items[i].key >> 56);
	const double N = rn_dmul((double)mass[p], s == 0 ? P.H_PER_MASS : P.HE_PER_MASS);
	float y = Y.yg[s][p];
	for (int j = i; j < M && run_of(items[j].key) == run; j++) {
		y = (float)rn_dsub((double)y, __ddiv_rn(rays[j].Nph, N));
		if (y < 0.0f) y = 0.0f;
	}
	Y.yg[s][p] = y;
}

// The emitters of the next tick: every particle on the hit lists of the
// tick's first nmark rays (its source rays and its first recombination ray).
__global__ void k_rec_mark(int R, const unsigned *__restrict__ count, const int64_t *__restrict__ off,
		const uint32_t *__restrict__ hit_ipar, const PsgBatchDev *__restrict__ B, int32_t *__restrict__ mark) {
	const int nmark = R + ((count[0] + count[1] + count[2]) > 0 ? 1 : 0);
	const int32_t tick = (int32_t)B->tick0;
	const int64_t end = off[nmark];
	for (int64_t h = off[0] + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; h < end;
			h += (int64_t)gridDim.x * blockDim.x)
		mark[hit_ipar[h]] = tick;
}

// Work space of the emission (S_RECW) for n particles and nspec species:
// draws -- the weights in caller order, their FP64 exclusive scan (n + 1),
// the scan's tile sums, the caller -> leaf map; threshold mode -- the
// flags of all species in caller order, their scan, its tile sums, the map.
struct RecWork {
	double *w, *ex, *tiles_d;
	uint32_t *flag;
	unsigned long long *pos, *tiles_u;
	uint32_t *leaf_of;
	size_t bytes;
};
RecWork rec_work(char *base, size_t n, int nspec, int threshold_mode) {
	RecWork r{};
	auto up = [](size_t x) { return (x + 255) & ~(size_t)255; };
	size_t o = 0;
	if (!threshold_mode) {
		r.w = (double *)(base + o); o = up(o + sizeof(double) * n);
		r.ex = (double *)(base + o); o = up(o + sizeof(double) * (n + 1));
		r.tiles_d = (double *)(base + o); o = up(o + sizeof(double) * (scan_tiles(n) + 1));
	} else {
		const size_t m = n * (size_t)nspec;
		r.flag = (uint32_t *)(base + o); o = up(o + sizeof(uint32_t) * m);
		r.pos = (unsigned long long *)(base + o); o = up(o + sizeof(unsigned long long) * (m + 1));
		r.tiles_u = (unsigned long long *)(base + o); o = up(o + sizeof(unsigned long long) * (scan_tiles(m) + 1));
	}
	r.leaf_of = (uint32_t *)(base + o); o = up(o + sizeof(uint32_t) * n);
	r.bytes = o;
	return r;
}

// Where the tick's rays end, in tick order: the draws' sort leaves them in
// the first or second half of S_RECK by its number of merge passes; the
// threshold mode places them in the first half.
RecItem *rec_sorted(psg_context *ctx, size_t ktot, int threshold_mode) {
	RecItem *items = (RecItem *)ctx->scratch[S_RECK].p;
	return (!threshold_mode && (dsort_passes(ktot) & 1)) ? items + ktot : items;
}

}  // namespace

// The tick's recombination rays into out (at most cap). One pass per
// species (HII; with helium also HeII and HeIII, loop.c:199): weights and
// draws into the species' part of the item array (unused entries stay all
// ones and sort last), then one merge sort of the whole array; or, with a
// threshold, flags in caller order, one scan and the placement. Launch
// sizes depend on n and the capacity only; the ray count lives in d_count
// (counters 11-13) and the kernels read it: no host read, so a tick can be
// captured. The tick number comes from B.
int psg_rec_prepare(psg_context *ctx) {
	const size_t n = ctx->n;
	const int threshold_mode = ctx->rec_nrec < 0;
	const int nspec = ctx->flags.h_only ? 1 : 3;
	const size_t kmax = threshold_mode ? n : (size_t)ctx->rec_nrec;     // per species
	const size_t ktot = kmax * nspec;
	const RecWork W = rec_work(nullptr, n, nspec, threshold_mode);
	if (!psg_scratch(ctx, S_RECW, W.bytes) || !psg_scratch(ctx, S_RECK, sizeof(RecItem) * 2 * ktot + 1024))
		return PSG_E_NOMEM;
	return PSG_OK;
}

int psg_rec_emit_enqueue(psg_context *ctx, const PsgBatchDev *B, psg_ray *out, unsigned long long *nlim,
		unsigned long long *recsum) {
	cudaStream_t st = ctx->stream;
	const size_t n = ctx->n;
	const PhysParams P = psg_phys_params(ctx);
	const int threshold_mode = ctx->rec_nrec < 0;
	const int nspec = ctx->flags.h_only ? 1 : 3;
	const size_t kmax = threshold_mode ? n : (size_t)ctx->rec_nrec;     // per species
	const size_t ktot = kmax * nspec;
	const RecWork W = rec_work((char *)ctx->scratch[S_RECW].p, n, nspec, threshold_mode);
	RecItem *items = (RecItem *)ctx->scratch[S_RECK].p;
	unsigned *d_count = (unsigned *)(ctx->d_counters + 11);      // [3]
	double *d_nph = (double *)(ctx->d_counters + 10);
	const RecState Y{{ctx->d_ygrec, ctx->d_ygrecHe1, ctx->d_ygrecHe2}};
	PSG_CUDA(cudaMemsetAsync(d_count, 0, sizeof(unsigned) * 4, st));
	if (!threshold_mode) {
		PSG_CUDA(cudaMemsetAsync(items, 0xff, sizeof(RecItem) * ktot, st));
		for (int s = 0; s < nspec; s++) {
			k_rec_weight<<<nblocks(n, 256), 256, 0, st>>>(n, B, ctx->d_srcmark, Y.yg[s], ctx->d_lambdaH,
					ctx->d_order, W.w, W.leaf_of);
			PSG_CHECK_LAUNCH();
			// cumulative weights: cdf[i] = ex[i + 1]
			PSG_CUDA(scan_enqueue(st, W.w, n, W.ex, W.tiles_d, AsDouble()));
			// streams: 4 the HII emitters, 7 and 8 those of HeII and HeIII
			k_rec_draw<<<nblocks(kmax, 128), 128, 0, st>>>(n, (int)kmax, s, s == 0 ? 4u : 6u + (uint32_t)s, W.ex + 1,
					B, ctx->rec_seed, W.leaf_of, items + s * kmax, d_count);
			PSG_CHECK_LAUNCH();
			ctx->launches += 5;
		}
		RecItem pad;
		memset(&pad, 0xff, sizeof(pad));
		PSG_CUDA(dsort_enqueue(st, items, items + ktot, ktot, pad, RecItemLess()));
		ctx->launches += 1 + dsort_passes(ktot);
	} else {
		for (int s = 0; s < nspec; s++) {
			k_rec_flag<<<nblocks(n, 256), 256, 0, st>>>(n, B, ctx->d_srcmark, Y.yg[s], ctx->rec_threshold,
					ctx->d_order, W.flag + (size_t)s * n, W.leaf_of);
			PSG_CHECK_LAUNCH();
			ctx->launches++;
		}
		PSG_CUDA(scan_enqueue(st, W.flag, n * nspec, W.pos, W.tiles_u, Widen()));
		k_rec_place<<<nblocks(n * nspec, 256), 256, 0, st>>>(n, nspec, W.flag, W.pos, W.leaf_of, items, d_count);
		PSG_CHECK_LAUNCH();
		ctx->launches += 4;
	}
	const RecItem *sorted = rec_sorted(ctx, ktot, threshold_mode);
	LteView L;
	L.cdf = ctx->d_lte;
	for (int s = 0; s < 3; s++) {
		L.freq_min[s] = ctx->lte_freq_min[s];
		L.freq_step[s] = ctx->lte_freq_step[s];
	}
	L.disabled = ctx->rec_disable_lte;
	const double length = ctx->boxsize * 2.0 * 0.1;     // MAX_REC_RAY_LENGTH, loop.c:169
	k_rec_rays<<<nblocks(ktot, 128), 128, 0, st>>>(d_count, nlim, recsum, sorted, B, ctx->rec_seed, ctx->d_psml,
			ctx->d_mass, Y,
			ctx->d_lambdaH, ctx->d_ie, P, L, length, out, d_nph);
	PSG_CHECK_LAUNCH();
	k_rec_purge<<<nblocks(ktot, 128), 128, 0, st>>>(d_count, sorted, out, ctx->d_mass, Y, P);
	PSG_CHECK_LAUNCH();
	ctx->launches += 2;
	return PSG_OK;
}

// The eager form: emission, then the count read back (one synchronisation).
static int emit_rec(psg_context *ctx, const PsgBatchDev *B, size_t cap, psg_ray *out, size_t *M_out) {
	int rc = psg_rec_prepare(ctx);
	if (!rc) rc = psg_rec_emit_enqueue(ctx, B, out, nullptr, nullptr);
	if (rc) return rc;
	unsigned cnt[3] = {0, 0, 0};
	PSG_CUDA(cudaMemcpyAsync(cnt, ctx->d_counters + 11, sizeof(unsigned) * 3, cudaMemcpyDeviceToHost, ctx->stream));
	PSG_CUDA(cudaStreamSynchronize(ctx->stream));
	ctx->host_syncs++;
	const size_t M = (size_t)cnt[0] + cnt[1] + cnt[2];
	if (M > cap) return psg_fail(ctx, PSG_E_OVERFLOW, "recombination rays: %zu > capacity %zu", M, cap);
	*M_out = M;
	return PSG_OK;
}

// The emitters of the next tick (k_rec_mark), R source rays.
int psg_rec_mark_enqueue(psg_context *ctx, size_t R, const PsgBatchDev *B) {
	k_rec_mark<<<4 * ctx->sms, 256, 0, ctx->stream>>>((int)R, (const unsigned *)(ctx->d_counters + 11),
			(const int64_t *)ctx->scratch[S_OFFSETS].p, (const uint32_t *)ctx->scratch[S_HIT_IPAR].p, B,
			ctx->d_srcmark);
	PSG_CHECK_LAUNCH();
	ctx->launches++;
	return PSG_OK;
}

// lte_init() / lte_fill() lte.c:30-72 for the three species (HI, HeI,
// HeII): 128 rows of log T from 3 to 10, 1024 energies from the threshold
// E_s up to 16 E_s; the weights sigma_s(E) E^3 exp(-(E - E_s)/kT) summed in
// order per row.
int psg_build_lte(psg_context *ctx, const psg_xs_table *xs) {
	const double th[3] = {ctx->u.HI_ENERGY, ctx->u.HEI_ENERGY, ctx->u.HEII_ENERGY};
	const int xsid[3] = {PSG_XS_HI, PSG_XS_HEI, PSG_XS_HEII};
	const double tstep = (10.0 - 3.0) / PSG_LTE_NLOGT;
	const size_t plane = (size_t)PSG_LTE_NLOGT * PSG_LTE_NFREQ;
	std::vector<double> cdf(3 * plane), freq(PSG_LTE_NFREQ);
	for (int s = 0; s < 3; s++) {
		const double fmin_ = th[s], fmax_ = 16.0 * th[s];
		const double fstep = (fmax_ - fmin_) / PSG_LTE_NFREQ;
		for (int j = 0; j < PSG_LTE_NFREQ; j++) freq[j] = fmin_ + fstep * j;
		for (int i = 0; i < PSG_LTE_NLOGT; i++) {
			const double logT = 3.0 + tstep * i;
			const double kT = ctx->u.BOLTZMANN * exp10(logT);
			double acc = 0.0;
			for (int j = 0; j < PSG_LTE_NFREQ; j++) {
				const double f = freq[j];
				acc += psg_xs_get(xs, xsid[s], f) * f * f * f * exp(-(f - fmin_) / kT);
				cdf[s * plane + (size_t)i * PSG_LTE_NFREQ + j] = acc;
			}
		}
		ctx->lte_freq_min[s] = fmin_;
		ctx->lte_freq_step[s] = fstep;
	}
	if (!ctx->d_lte) PSG_CUDA(cudaMalloc(&ctx->d_lte, sizeof(double) * cdf.size()));
	PSG_CUDA(cudaMemcpy(ctx->d_lte, cdf.data(), sizeof(double) * cdf.size(), cudaMemcpyHostToDevice));
	return PSG_OK;
}

int psg_run_ticks_rec(psg_context *ctx, const psg_ray *d_rays, size_t R, size_t K, int64_t first_tick,
		double tick_time, psg_tick_stats *stats) {
	cudaStream_t st = ctx->stream;
	const size_t cap = (ctx->rec_nrec > 0 ? (size_t)ctx->rec_nrec : ctx->rec_nrec < 0 ? ctx->n : 0) *
			(ctx->flags.h_only ? 1 : 3);
	if (R + cap >= (size_t)INT32_MAX) return psg_fail(ctx, PSG_E_OVERFLOW, "psg_run_ticks: batch too large");
	psg_ray *buf = (psg_ray *)psg_scratch(ctx, S_RECRAYS, sizeof(psg_ray) * (R + cap));
	if (!buf) return PSG_E_NOMEM;
	double *d_nph = (double *)(ctx->d_counters + 10);
	PSG_CUDA(cudaMemsetAsync(d_nph, 0, sizeof(double), st));
	psg_tick_stats acc{}, one{};
	double rec_rays = 0.0, syncs = 0.0;
	long launches = 0;
	if (ctx->rec_nrec > 0 && ctx->use_graphs && !ctx->timing) {
		// the ticks replayed from a captured tick, no host read between them
		const int rc = psg_run_ticks_rec_graph(ctx, d_rays, R, K, first_tick, tick_time, stats);
		if (rc != PSG_RETRY) return rc;
	}
	for (size_t k = 0; k < K; k++) {
		const int64_t tick = first_tick + (int64_t)k;
		PSG_CUDA(cudaMemcpyAsync(buf, d_rays + k * R, sizeof(psg_ray) * R, cudaMemcpyDeviceToDevice, st));
		ctx->launches = 0;
		ctx->host_syncs = 0;
		size_t M = 0;
		if (ctx->rec_nrec != 0) {      // (no rays at the first tick, loop.c:197: k_rec_draw, k_rec_flag)
			k_set_batch_rec<<<1, 1, 0, st>>>(ctx->d_batch, tick, tick_time, buf, d_rays, (int64_t)k);
			PSG_CHECK_LAUNCH();
			const int rc = emit_rec(ctx, ctx->d_batch, cap, buf + R, &M);
			if (rc) return rc;
		}
		const long emit_launches = ctx->launches;
		syncs += (double)ctx->host_syncs;
		ctx->rec_last = M;
		ctx->rec_last_R = R;
		ctx->rec_last_kmax = cap;
		ctx->rec_last_threshold = ctx->rec_nrec < 0;
		rec_rays += (double)M;
		int rc = psg_run_ticks_core(ctx, buf, R + M, 1, tick, tick_time, &one);
		if (rc) return rc;
		if (ctx->rec_nrec == 0) PSG_CUDA(cudaMemsetAsync(ctx->d_counters + 11, 0, 4 * sizeof(unsigned), st));
		rc = psg_rec_mark_enqueue(ctx, R, ctx->d_batch);
		if (rc) return rc;
		launches += emit_launches + (long)one.launches + 1;
		acc.hits += one.hits;
		acc.saturated += one.saturated;
		acc.active += one.active;
		acc.lost_photons += one.lost_photons;
		acc.trace_ms += one.trace_ms;
		syncs += one.host_syncs;
		acc.tick_ms += one.tick_ms;
		for (int g = 0; g < PSG_K_NKERNELS; g++) {
			acc.kernel_ms[g] += one.kernel_ms[g];
			acc.kernel_launches[g] += one.kernel_launches[g];
		}
	}
	double nph = 0.0;
	PSG_CUDA(cudaMemcpyAsync(&nph, d_nph, sizeof(double), cudaMemcpyDeviceToHost, st));
	PSG_CUDA(cudaStreamSynchronize(st));
	ctx->launches = launches;
	if (stats) {
		acc.launches = (double)launches;
		acc.host_syncs = syncs + 1.0;
		acc.rec_rays = rec_rays;
		acc.rec_photons = nph;
		*stats = acc;
	}
	return PSG_OK;
}

extern "C" int psg_set_recombination(psg_context *ctx, int nrec, double threshold, int disable_lte,
		uint64_t seed) {
	if (!ctx) return PSG_E_INVAL;
	if (!(threshold >= 0.0)) return psg_fail(ctx, PSG_E_INVAL, "psg_set_recombination: threshold must be >= 0");
	if (nrec >= (1 << 24)) return psg_fail(ctx, PSG_E_INVAL, "psg_set_recombination: nrec must be below 2^24");
	ctx->rec_nrec = nrec;
	ctx->rec_threshold = threshold;
	ctx->rec_disable_lte = disable_lte != 0;
	ctx->rec_seed = seed;
	return PSG_OK;
}

extern "C" int psg_get_rec_rays(psg_context *ctx, psg_ray *rays, int64_t *ipar, int32_t *type, size_t cap,
		size_t *n) {
	if (!ctx) return PSG_E_INVAL;
	if (!n) return psg_fail(ctx, PSG_E_INVAL, "psg_get_rec_rays: null count");
	*n = ctx->rec_last;
	if (ctx->rec_last == 0 || (!rays && !ipar && !type)) return PSG_OK;
	if (cap < ctx->rec_last) return psg_fail(ctx, PSG_E_INVAL, "psg_get_rec_rays: %zu rays, capacity %zu", ctx->rec_last, cap);
	PSG_CUDA(cudaSetDevice(ctx->device));
	const size_t M = ctx->rec_last;
	const size_t kmax = ctx->rec_last_kmax;
	if (rays)
		PSG_CUDA(cudaMemcpyAsync(rays, (psg_ray *)ctx->scratch[S_RECRAYS].p + ctx->rec_last_R, sizeof(psg_ray) * M,
				cudaMemcpyDeviceToHost, ctx->stream));
	std::vector<RecItem> items(M);
	if (ipar || type)
		PSG_CUDA(cudaMemcpyAsync(items.data(), rec_sorted(ctx, kmax, ctx->rec_last_threshold), sizeof(RecItem) * M,
				cudaMemcpyDeviceToHost, ctx->stream));
	PSG_CUDA(cudaStreamSynchronize(ctx->stream));
	for (size_t i = 0; i < M; i++) {
		if (ipar) ipar[i] = (int64_t)((items[i].key >> 24) & 0xFFFFFFFFull);
		if (type) type[i] = (int32_t)(items[i].key >> 56);
	}
	return PSG_OK;
}
