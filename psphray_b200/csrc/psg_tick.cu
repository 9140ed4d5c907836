// Ticks: deposit (loop.c:388-608), merge (loop.c:610-645) and update
// (loop.c:647-776) for many ticks whose rays are traced in one batch.
//
// Hit lists depend only on geometry, so all rays of a batch of ticks are
// traced together. Before the tick loop the hits are put in a by-particle
// order ((tick, ipar, hit) sorted: the slot order, vals[slot] = hit), which
// turns the reference's merge into the runs of equal (tick, ipar) and its
// float atomics into a fixed-order FP64 sum per particle. Then per tick:
//   deposit: a group of threads per ray (a warp, a 128-thread quarter or a
//     512-thread block) walks its sorted hits; optical depths are summed with
//     an FP64 group scan, the transmitted photons before each hit are
//     TM*exp(-scan), absorbed = TM_j*(1-e^-tau_j); the first hit whose
//     absorption exceeds its neutral atoms (the cap of loop.c:482-485) or
//     after which TM/Nph < 1e-10 (loop.c:585) is settled on its own and the
//     scan restarts after it. Each hit writes photons/NH at its own index (in
//     ray order), or -1 when the reference would not deposit there;
//   update: every particle hit in the tick sums its deposits in slot order
//     (gathered through vals) and advances (lambdaH, ie) by the step since
//     its last hit.
#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "psg_internal.cuh"
#include "psg_bsort.cuh"
#include "psg_scan.cuh"
#include "psg_helium.cuh"
#include "psg_solve.cuh"
#include "psg_surrogate.cuh"

PhysParams psg_phys_params(const psg_context *ctx) {
	PhysParams P{};
	P.ar = ctx->d_ar;
	P.ar_ni = ctx->d_ar_ni;
	for (int c = 0; c < 8; c++) P.ar_ni_scale[c] = ctx->ar_ni_scale[c];
	P.ar_all = ctx->d_ar_all;
	for (int c = 0; c < PSG_AR_NCOLS; c++) P.ar_all_scale[c] = ctx->ar_all_scale[c];
	P.ar_step = ctx->ar_step;
	P.ar_nrows = ctx->ar_nrows;
	P.ar_min = ctx->ar_min;
	P.ar_step_inv = ctx->ar_step_inv;
	P.ar_min_f = (float)ctx->ar_min;
	P.ar_step_f = (float)ctx->ar_step;
	P.ar_step_inv_f = (float)ctx->ar_step_inv;
	P.xs = ctx->d_xs;
	P.xs_nrows = ctx->xs_nrows;
	P.xs_min = ctx->xs_min;
	P.xs_step_inv = ctx->xs_step_inv;
	P.xs_cut_HI = ctx->xs_cut_HI;
	P.kernel = ctx->d_kernel;
	P.kernel_n = ctx->kernel_n;
	P.H_PER_MASS = ctx->u.H_PER_MASS;
	P.HI_ENERGY = ctx->u.HI_ENERGY;
	P.MPROTON_OVER_BOLTZMANN = ctx->u.MPROTON_OVER_BOLTZMANN;
	P.BOLTZMANN_OVER_MPROTON = ctx->u.BOLTZMANN_OVER_MPROTON;
	P.hmf = ctx->u.hmf;
	P.hemf = ctx->u.hemf;
	// lambda_to_ye() psystem.h:134-138 with lambdaHeI = lambdaHeII = 0
	P.he_e = ctx->u.hemf / ctx->u.hmf * 0.25 * (0.0 + 2 * (1.0 - 0.0 - 0.0));
	P.isothermal = ctx->flags.isothermal;
	P.on_the_spot = ctx->flags.on_the_spot;
	P.adiabatic = ctx->flags.adiabatic;
	P.euler = ctx->flags.euler;
	P.ygrec = ctx->flags.on_the_spot ? nullptr : ctx->d_ygrec;
	P.xs_cut_HeI = ctx->xs_cut_HeI;
	P.xs_cut_HeII = ctx->xs_cut_HeII;
	P.h_only = ctx->flags.h_only;
	P.secondary = ctx->flags.secondary_ionization;
	P.HE_PER_MASS = ctx->u.HE_PER_MASS;
	P.HEI_ENERGY = ctx->u.HEI_ENERGY;
	P.HEII_ENERGY = ctx->u.HEII_ENERGY;
	P.lamHeI = ctx->d_lamHeI;
	P.lamHeII = ctx->d_lamHeII;
	P.ygrecHe1 = ctx->flags.on_the_spot ? nullptr : ctx->d_ygrecHe1;
	P.ygrecHe2 = ctx->flags.on_the_spot ? nullptr : ctx->d_ygrecHe2;
	P.gcarry = ctx->d_gcarry;
	P.gcarryHe1 = ctx->d_gcarryHe1;
	P.gcarryHe2 = ctx->d_gcarryHe2;
	// secion_init() secion.c:75-86
	P.si = ctx->d_si;
	P.si_min1 = 10 * ctx->u.EV;
	P.si_step1 = (200 * ctx->u.EV - P.si_min1) / PSG_SECION_NE;
	P.si_step1_inv = 1.0 / P.si_step1;
	P.si_min2 = -8;
	P.si_step2 = (0.0 - P.si_min2) / PSG_SECION_NX;
	P.si_step2_inv = 1.0 / P.si_step2;
	return P;
}

namespace {

inline unsigned blocks(size_t n, int bs) { return (unsigned)((n + bs - 1) / bs); }


// ---- the by-particle order without a key sort ------------------------------
// The slots of a batch: every hit of tick t on particle p gets a place in the
// (t, p, hit index) order. Counting instead of sorting: per (t, p) key the
// number of hits (atomics on counters zeroed per batch), one exclusive scan
// of the (count, count > 0) pairs over the K*N keys gives each key its first
// slot and its active-particle index, a second pass places every hit in its
// key's run (any order), and the runs longer than 32 are sorted into
// hit-index order -- the order a stable key sort gives; the per-particle
// sums read the shorter ones in hit order by selection (next_in_run), so
// every sum adds in a fixed order.

// one warp per ray: count the ray's hits per key (tick * N + particle)
__global__ void k_slot_count(size_t nray, int R, uint32_t N, const int64_t *__restrict__ off,
		const uint32_t *__restrict__ ipar, uint32_t *__restrict__ cnt) {
	const size_t r = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) / 32;
	const int lane = threadIdx.x & 31;
	if (r >= nray) return;
	const size_t base = (r / (size_t)R) * N;
	for (int64_t h = off[r] + lane; h < off[r + 1]; h += 32) atomicAdd(&cnt[base + ipar[h]], 1u);
}

// the active (tick, particle) pairs in key order: their particle and first
// slot, the first pair of every tick and the totals; and every key's
// counter set to the end of its run, for the placement below
__global__ void k_act_build(size_t KN, uint32_t N, int K, const unsigned long long *__restrict__ base,
		uint32_t *__restrict__ act_ipar, uint32_t *__restrict__ act_seg, int32_t *__restrict__ tick_act,
		unsigned long long *__restrict__ nact_out, uint32_t *__restrict__ cnt) {
	for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < KN; k += (size_t)gridDim.x * blockDim.x) {
		const unsigned long long b0 = base[k], b1 = base[k + 1];
		const uint32_t a = (uint32_t)(b0 >> 32);
		if ((uint32_t)(b1 >> 32) != a) {
			act_ipar[a] = (uint32_t)(k % N);
			act_seg[a] = (uint32_t)b0;
			cnt[k] = (uint32_t)b1;
		}
		if (k % N == 0) tick_act[k / N] = (int32_t)a;
	}
	if (blockIdx.x == 0 && threadIdx.x == 0) {
		const unsigned long long tot = base[KN];
		const uint32_t nact = (uint32_t)(tot >> 32);
		tick_act[K] = (int32_t)nact;
		act_seg[nact] = (uint32_t)tot;
		atomicAdd(nact_out, (unsigned long long)nact);     // over the call's batches
	}
}

// one warp per ray: every hit into its key's run, at the slot its counter
// (the run's end, counting down) gives; vals[slot] = the hit. The counters
// are left at the runs' first slots (zeroed before the next batch).
__global__ void k_slot_place(size_t nray, int R, uint32_t N, const int64_t *__restrict__ off,
		const uint32_t *__restrict__ ipar, uint32_t *__restrict__ cnt, uint32_t *__restrict__ vals) {
	const size_t r = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) / 32;
	const int lane = threadIdx.x & 31;
	if (r >= nray) return;
	const size_t kb = (r / (size_t)R) * N;
	for (int64_t h = off[r] + lane; h < off[r + 1]; h += 32)
		vals[atomicSub(&cnt[kb + ipar[h]], 1u) - 1u] = (uint32_t)h;
}

// Runs longer than the tuner's run_short (particles next to a source), in three tiers: up to
// SLOT_WARP_MAX hits a warp each (bitonic sort in the warp's part of
// shared memory); up to SLOT_MID_MAX a 256-thread block each (bitonic in
// shared memory); longer ones a 1024-thread block each, bitonic in shared
// memory up to cap_pow2 (the tick's rays rounded up to a power of two, at
// most SLOT_LONG_MAX) and merge-sorted in global memory beyond that (more
// than SLOT_LONG_MAX rays of one tick on one particle), with the upper half
// of vals (from half) as scratch. The two block tiers take their runs from
// lists of their own.
#define RUN_SHORT 16         // the longest run that may be left unsorted (psg_tune.run_short: 4, 8 or 16)
#define RUN_THREAD 32        // runs up to this many hits are summed by a thread, longer ones by a warp
#define SLOT_WARP_MAX 256
#define SLOT_MID_MAX 2048
#define SLOT_LONG_MAX 32768
#define SLOT_WARPS 8
struct U32Less {
	__device__ __forceinline__ bool operator()(uint32_t x, uint32_t y) const { return x < y; }
};
__global__ void __launch_bounds__(32 * SLOT_WARPS) k_slot_canon_warp(const int32_t *__restrict__ tick_long, int K,
		const uint32_t *__restrict__ long_act, const uint32_t *__restrict__ act_seg, uint32_t *__restrict__ vals) {
	__shared__ uint32_t sv_all[SLOT_WARPS][SLOT_WARP_MAX];
	uint32_t *sv = sv_all[threadIdx.x >> 5];
	const int lane = threadIdx.x & 31;
	const int ne = tick_long[K];
	for (int e = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); e < ne; e += (int)((gridDim.x * blockDim.x) >> 5)) {
		const uint32_t a = long_act[e];
		const uint32_t s0 = act_seg[a], n = act_seg[a + 1] - s0;
		if (n > SLOT_WARP_MAX) continue;
		int P = 16;
		while (P < (int)n) P <<= 1;
		for (int i = lane; i < P; i += 32) sv[i] = i < (int)n ? vals[s0 + i] : 0xFFFFFFFFu;
		__syncwarp();
		for (int k = 2; k <= P; k <<= 1) {
			for (int j = k >> 1; j > 0; j >>= 1) {
				for (int i = lane; i < P; i += 32) {
					const int ixj = i ^ j;
					if (ixj > i) {
						const uint32_t x = sv[i], y = sv[ixj];
						if ((x > y) == ((i & k) == 0)) {
							sv[i] = y;
							sv[ixj] = x;
						}
					}
				}
				__syncwarp();
			}
		}
		for (int i = lane; i < (int)n; i += 32) vals[s0 + i] = sv[i];
		__syncwarp();
	}
}
// P <= PMAX elements of sv sorted by the block (bitonic); callers sync
// before, the last stage syncs after
template <int NT>
__device__ __forceinline__ void block_bitonic_u32(uint32_t *sv, int P) {
	for (int k = 2; k <= P; k <<= 1) {
		for (int j = k >> 1; j > 0; j >>= 1) {
			for (int i = threadIdx.x; i < P; i += NT) {
				const int ixj = i ^ j;
				if (ixj > i) {
					const uint32_t x = sv[i], y = sv[ixj];
					if ((x > y) == ((i & k) == 0)) {
						sv[i] = y;
						sv[ixj] = x;
					}
				}
			}
			__syncthreads();
		}
	}
}
__global__ void __launch_bounds__(256) k_slot_canon_mid(const uint32_t *__restrict__ list,
		const unsigned *__restrict__ count, const uint32_t *__restrict__ act_seg, uint32_t *__restrict__ vals) {
	__shared__ uint32_t sv[SLOT_MID_MAX];
	const int ne = (int)*count;
	for (int e = blockIdx.x; e < ne; e += gridDim.x) {
		const uint32_t a = list[e];
		const uint32_t s0 = act_seg[a], n = act_seg[a + 1] - s0;
		int P = 2 * SLOT_WARP_MAX;
		while (P < (int)n) P <<= 1;
		for (int i = threadIdx.x; i < P; i += 256) sv[i] = i < (int)n ? vals[s0 + i] : 0xFFFFFFFFu;
		__syncthreads();
		block_bitonic_u32<256>(sv, P);
		for (int i = threadIdx.x; i < (int)n; i += 256) vals[s0 + i] = sv[i];
		__syncthreads();
	}
}
__global__ void __launch_bounds__(1024) k_slot_canon_long(const uint32_t *__restrict__ vl_list,
		const unsigned *__restrict__ vl_count, const uint32_t *__restrict__ act_seg, uint32_t *__restrict__ vals,
		int cap_pow2, size_t half) {
	extern __shared__ uint32_t sv[];
	const int ne = (int)*vl_count;
	for (int e = blockIdx.x; e < ne; e += gridDim.x) {
		const uint32_t a = vl_list[e];
		const uint32_t s0 = act_seg[a], n = act_seg[a + 1] - s0;
		if ((int)n > cap_pow2) {      // (shared memory holds at least the merge sort's 2048-entry tile)
			const uint32_t *f = block_sort_global<1024>(vals + s0, vals + half + s0, (int64_t)n, sv, 0xFFFFFFFFu,
					U32Less());
			for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) vals[s0 + i] = f[i];
			__syncthreads();
			continue;
		}
		int P = 1;
		while (P < (int)n) P <<= 1;
		for (int i = threadIdx.x; i < P; i += blockDim.x) sv[i] = i < (int)n ? vals[s0 + i] : 0xFFFFFFFFu;
		__syncthreads();
		block_bitonic_u32<1024>(sv, P);
		for (int i = threadIdx.x; i < (int)n; i += blockDim.x) vals[s0 + i] = sv[i];
		__syncthreads();
	}
}

__device__ __forceinline__ bool below_cutoff(double TM, double Nph) {
	return TM < 0.0 || __ddiv_rn(TM, Nph) < 1e-10;
}

// Deposit of one ray by a group of NT threads (a warp, a 128-thread quarter
// or a whole block): hits are taken NT at a time; optical depths are summed
// with an FP64 scan over the group; the first hit whose absorption exceeds
// its neutral atoms (loop.c:482-485) or after which TM/Nph < 1e-10
// (loop.c:585) is found with a group min, settled by its own thread, and the
// scan restarts after it (or, in the AFF form, the rest of the step goes to
// settle_capped()). Transmitted photons before hit j are
// TM*exp(-(sum of earlier tau)); after it, TM_j minus the absorbed photons,
// as loop.c:580 updates TM. Each hit writes photons/NH at its index, or -1
// where the reference deposits nothing. wsum and wb carry the per-warp scan
// totals (wb: the affine maps' offsets).
struct DepShared {
	double wsum[32];
	double wb[32];
	double tm;
	int first;
};

// The threads of one ray: a warp, a 128-thread quarter of a block (named
// barrier `bar`, 1..4) or the whole block (bar 0).
template <int NT>
__device__ __forceinline__ void group_sync(int bar) {
	if (NT == 32) __syncwarp();
	else if (bar == 0) __syncthreads();
	else asm volatile("bar.sync %0, %1;" ::"r"(bar), "n"(NT) : "memory");
}

// One hit's deposits sit together, nacc doubles per hit (photons/NH; with
// heat the heat; with helium yGdepHeI and yGdepHeII), at the hit's index:
// a ray's group stores contiguously, and the by-particle sums gather one
// 8- to 32-byte record per deposit through the slot order.
__device__ __forceinline__ void acc_store(double *__restrict__ acc, int nacc, uint32_t s, double y, double heat,
		double y1, double y2) {
	if (nacc == 4) {
		double2 *a = reinterpret_cast<double2 *>(acc) + 2 * (size_t)s;
		a[0] = make_double2(y, heat);
		a[1] = make_double2(y1, y2);
	} else if (nacc == 2) {
		reinterpret_cast<double2 *>(acc)[s] = make_double2(y, heat);
	} else {
		acc[s] = y;
	}
}

// Past a capped hit f the step mixes capped hits, which take TM to
// TM - NHI (loop.c:482-485, 580), and uncapped ones, TM to TM*exp(-tau):
// affine maps, whose composition is associative. A group scan of the maps
// gives TM before every hit for a guessed capped/uncapped pattern; the hits
// before the first whose decision (or the 1e-10 cut) disagrees with the
// guess are settled, that one is settled from its exact TM, and the next
// pass guesses from this pass's decisions. TM changes slowly along a capped
// run, so a step settles in a few passes instead of one per capped hit.
// Called by every thread of the group with start = f + 1 and TM after f;
// returns with the step settled (or the ray done). The deposit takes this
// form (AFF) when the previous batch capped more than 1e-3 of its hits: on
// a ray with few capped hits, its registers slow the common path.
template <int NT>
__device__ __forceinline__ void settle_capped(int t, bool valid, double tau, double NHI, double NH_inv, double Nph,
		int start, double &TM, bool &done, double &delta, unsigned &nsat, DepShared &sh, int bar) {
	const int lane = t & 31, wid = t >> 5;
	constexpr int NW = NT / 32;
	const double m1 = (valid && tau != 0.0) ? -expm1(-tau) : 0.0;
	bool pcap = valid && t >= start && tau != 0.0 && TM * m1 > NHI;
	while (start < NT) {
		const bool pb = valid && t >= start && tau != 0.0;
		double A = 1.0, B = 0.0;            // this hit's map, TM -> A*TM + B
		if (pb) {
			if (pcap) B = -NHI;
			else A = 1.0 - m1;
		}
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			const double pa = __shfl_up_sync(0xffffffffu, A, o);
			const double pv = __shfl_up_sync(0xffffffffu, B, o);
			if (lane >= o) {
				B = A * pv + B;
				A = A * pa;
			}
		}
		// the maps of the hits before this one: the lower lanes', after
		// the earlier warps'
		double xa = __shfl_up_sync(0xffffffffu, A, 1), xb = __shfl_up_sync(0xffffffffu, B, 1);
		if (lane == 0) { xa = 1.0; xb = 0.0; }
		double ta = A, tb = B;               // the whole step's map
		if (NW > 1) {
			if (lane == 31) { sh.wsum[wid] = A; sh.wb[wid] = B; }
			if (t == 0) sh.first = NT;
			group_sync<NT>(bar);
			double ea = 1.0, eb = 0.0;
			ta = 1.0;
			tb = 0.0;
#pragma unroll
			for (int k = 0; k < NW; k++) {
				const double wa = sh.wsum[k], wb = sh.wb[k];
				if (k < wid) {
					eb = wa * eb + wb;
					ea = wa * ea;
				}
				tb = wa * tb + wb;
				ta = wa * ta;
			}
			xb = xa * eb + xb;
			xa = xa * ea;
		} else {
			ta = __shfl_sync(0xffffffffu, A, 31);
			tb = __shfl_sync(0xffffffffu, B, 31);
		}
		double TMj = 0.0, absorb = 0.0, after = 0.0;
		bool cap = false, bad = false;
		if (pb) {
			TMj = xa * TM + xb;
			absorb = TMj * m1;
			cap = absorb > NHI;
			after = cap ? TMj - NHI : TMj - absorb;
			bad = (cap != pcap) || below_cutoff(after, Nph);
		}
		int m;
		if (NW == 1) {
			const unsigned ev = __ballot_sync(0xffffffffu, bad);
			m = ev ? __ffs(ev) - 1 : NT;
		} else {
			if (bad) atomicMin(&sh.first, t);
			group_sync<NT>(bar);
			m = sh.first;
		}
		if (pb && t <= m) {        // the settled hits, and hit m from its exact TM
			delta = rn_dmul(cap ? NHI : absorb, NH_inv);
			if (cap) nsat++;
		}
		if (m == NT) {
			TM = ta * TM + tb;
			group_sync<NT>(bar);       // shared words are rewritten by the next scan
			break;
		}
		if (NW == 1) {
			TM = __shfl_sync(0xffffffffu, after, m);
		} else {
			if (t == m) sh.tm = after;
			group_sync<NT>(bar);
			TM = sh.tm;
		}
		start = m + 1;
		pcap = cap;
		group_sync<NT>(bar);
		if (below_cutoff(TM, Nph)) {
			done = true;
			break;
		}
	}
}

template <int NT, bool AFF>
__device__ void deposit_ray(const psg_ray &ray, int64_t h0, int64_t h1, int t,
		const uint32_t *__restrict__ hipar, const double *__restrict__ hkern,
		const double *__restrict__ lambdaH, const float *__restrict__ mass, const PhysParams &P, int want_heat,
		double *__restrict__ acc, DepShared &sh, unsigned &nsat, double &lost, int bar) {
	const int lane = t & 31, wid = t >> 5;
	constexpr int NW = NT / 32;
	const double Nph = ray.Nph;
	const double freq = ray.freq;
	const bool skip_ray = (Nph == 0.0);
	const double sigma = xs_get_HI(P, freq);
	const double heat_factor = rn_dmul(P.H_PER_MASS, fdim(freq, P.HI_ENERGY));
	double TM = Nph;
	bool done = skip_ray;
	// the next step's loads are issued one step ahead
	double np_kern = 0.0, np_lam = 0.0;
	float np_mass = 1.0f;
	{
		const int64_t h = h0 + t;
		if (h < h1) {
			const uint32_t p = hipar[h];
			np_kern = hkern[h];
			if (!done) { np_lam = lambdaH[p]; np_mass = mass[p]; }
		}
	}
	for (int64_t base = h0; base < h1; base += NT) {
		const int64_t h = base + t;
		const bool valid = h < h1;
		const double kern_c = np_kern, lam_c = np_lam;
		const float mass_c = np_mass;
		const uint32_t slot_c = (uint32_t)h;      // (a hit's deposits sit at its own index)
		{
			const int64_t hn = h + NT;
			if (hn < h1) {
				const uint32_t p = hipar[hn];
				np_kern = hkern[hn];
				if (!done) { np_lam = lambdaH[p]; np_mass = mass[p]; }
			}
		}
		double tau = 0.0, NHI = 0.0, NH_inv = 0.0, delta = -1.0;
		if (valid && !done) {
			const double NH = rn_dmul((double)mass_c, P.H_PER_MASS);
			NHI = rn_dmul(lam_c, NH);
			tau = rn_dmul(sigma, rn_dmul(kern_c, NHI));
			NH_inv = __ddiv_rn(1.0, NH);
		}
		int start = 0;
		while (!done && start < NT) {
			const bool part = valid && t >= start && tau != 0.0;
			const double my_tau = part ? tau : 0.0;
			double wi = my_tau;
#pragma unroll
			for (int o = 1; o < 32; o <<= 1) {
				const double v = __shfl_up_sync(0xffffffffu, wi, o);
				if (lane >= o) wi += v;
			}
			double woff = 0.0, total;
			if (NW == 1) {
				total = __shfl_sync(0xffffffffu, wi, 31);
			} else {
				if (lane == 31) sh.wsum[wid] = wi;
				if (t == 0) sh.first = NT;
				group_sync<NT>(bar);
				total = 0.0;
#pragma unroll
				for (int k = 0; k < NW; k++) {
					const double v = sh.wsum[k];
					if (k < wid) woff += v;
					total += v;
				}
			}
			double TMj = 0.0, absorb = 0.0, TMafter = 0.0;
			bool capped = false, cut = false;
			if (part) {
				const double excl = (woff + wi) - my_tau;
				TMj = TM * exp(-excl);
				absorb = TMj * -expm1(-my_tau);
				TMafter = TMj - absorb;
				capped = absorb > NHI;
				cut = below_cutoff(TMafter, Nph);
			}
			int f;
			if (NW == 1) {
				const unsigned ev = __ballot_sync(0xffffffffu, capped || cut);
				f = ev ? __ffs(ev) - 1 : NT;
			} else {
				if (capped || cut) atomicMin(&sh.first, t);
				group_sync<NT>(bar);
				f = sh.first;
			}
			if (part && t < f) delta = rn_dmul(absorb, NH_inv);
			if (f == NT) {
				TM = TM * exp(-total);
				group_sync<NT>(bar);       // shared words are rewritten by the next step
				break;
			}
			double TMnew = 0.0;
			if (t == f) {
				TMnew = TMafter;
				if (capped) {
					absorb = NHI;
					TMnew = TMj - NHI;
					nsat++;
				}
				delta = rn_dmul(absorb, NH_inv);
				if (NW > 1) sh.tm = TMnew;
			}
			if (NW == 1) {
				TM = __shfl_sync(0xffffffffu, TMnew, f);
			} else {
				group_sync<NT>(bar);
				TM = sh.tm;
			}
			if (below_cutoff(TM, Nph)) done = true;
			start = f + 1;
			group_sync<NT>(bar);
			if (AFF && !done) {
				// f was capped: the rest of the step through the affine-map scan
				settle_capped<NT>(t, valid, tau, NHI, NH_inv, Nph, start, TM, done, delta, nsat, sh, bar);
				break;
			}
		}
		if (valid) {
			acc_store(acc, want_heat ? 2 : 1, slot_c, delta,
					want_heat && delta >= 0.0 ? rn_dmul(heat_factor, delta) : 0.0, 0.0, 0.0);
		}
	}
	if (t == 0 && !skip_ray) lost += TM;
}

// The same with helium and/or secondary ionisation (loop.c:409-567): the
// scan runs over the sum of the three species' optical depths; a hit
// absorbs tau_s/tausum of the photons per species, each capped at its
// atoms (loop.c:476-505); it writes yGdepHI, heat, yGdepHeI and yGdepHeII
// increments (nacc of them per hit), with the secondary
// ionisation and heating of loop.c:513-552 (whose HeII terms the
// reference's statements drop, loop.c:523,542).
template <int NT>
__device__ void deposit_ray_gen(const psg_ray &ray, int64_t h0, int64_t h1, int t,
		const uint32_t *__restrict__ hipar, const double *__restrict__ hkern,
		const double *__restrict__ lambdaH, const float *__restrict__ mass, const PhysParams &P, int want_heat,
		double *__restrict__ acc, int nacc, DepShared &sh, unsigned &nsat, double &lost, int bar) {
	const int lane = t & 31, wid = t >> 5;
	constexpr int NW = NT / 32;
	const double Nph = ray.Nph;
	const double freq = ray.freq;
	const bool skip_ray = (Nph == 0.0);
	const double sigma = xs_get_HI(P, freq);
	const double sHeI = xs_get_s(P, 1, freq), sHeII = xs_get_s(P, 2, freq);
	const double dE0 = fdim(freq, P.HI_ENERGY), dE1 = fdim(freq, P.HEI_ENERGY), dE2 = fdim(freq, P.HEII_ENERGY);
	const double hf0 = P.H_PER_MASS * dE0, hf1 = P.HE_PER_MASS * dE1, hf2 = P.HE_PER_MASS * dE2;
	double TM = Nph;
	bool done = skip_ray;
	// the next step's loads are issued one step ahead
	double np_kern = 0.0, np_lam = 0.0, np_l1 = 0.0, np_l2 = 0.0;
	float np_mass = 1.0f;
	{
		const int64_t h = h0 + t;
		if (h < h1) {
			const uint32_t p = hipar[h];
			np_kern = hkern[h];
			if (!done) { np_lam = lambdaH[p]; np_mass = mass[p]; np_l1 = P.lamHeI[p]; np_l2 = P.lamHeII[p]; }
		}
	}
	for (int64_t base = h0; base < h1; base += NT) {
		const int64_t h = base + t;
		const bool valid = h < h1;
		const double kern_c = np_kern, lam_c = np_lam, l1_c = np_l1, l2_c = np_l2;
		const float mass_c = np_mass;
		const uint32_t slot_c = (uint32_t)h;      // (a hit's deposits sit at its own index)
		{
			const int64_t hn = h + NT;
			if (hn < h1) {
				const uint32_t p = hipar[hn];
				np_kern = hkern[hn];
				if (!done) { np_lam = lambdaH[p]; np_mass = mass[p]; np_l1 = P.lamHeI[p]; np_l2 = P.lamHeII[p]; }
			}
		}
		// species s = 0 HI, 1 HeI, 2 HeII: atoms N_s, optical depth t_s
		double tau = 0.0, NHI = 0.0, NH_inv = 0.0, delta = -1.0;
		double N1 = 0.0, N2 = 0.0, t0 = 0.0, t1 = 0.0, t2 = 0.0, NHe_inv = 0.0, xe = 0.0;
		double d0 = 0.0, d1 = 0.0, d2 = 0.0;
		bool he = false;
		if (valid && !done) {
			const double NH = (double)mass_c * P.H_PER_MASS;
			const double NHe = (double)mass_c * P.HE_PER_MASS;
			NHI = lam_c * NH;
			t0 = sigma * (kern_c * NHI);
			tau = 0.0 + t0;
			he = !P.h_only && NHe != 0.0;
			if (he) {
				N1 = l1_c * NHe;
				t1 = sHeI * (kern_c * N1);
				tau += t1;
				N2 = l2_c * NHe;
				t2 = sHeII * (kern_c * N2);
				tau += t2;
			}
			NH_inv = 1.0 / NH;
			NHe_inv = 1.0 / NHe;
			xe = ye_he(P, lam_c, l1_c, l2_c) * NH / (NH + NHe);     // loop.c:512-513
			if (xe > 1.0) xe = 1.0;
		}
		int start = 0;
		while (!done && start < NT) {
			const bool part = valid && t >= start && tau != 0.0;
			const double my_tau = part ? tau : 0.0;
			double wi = my_tau;
#pragma unroll
			for (int o = 1; o < 32; o <<= 1) {
				const double v = __shfl_up_sync(0xffffffffu, wi, o);
				if (lane >= o) wi += v;
			}
			double woff = 0.0, total;
			if (NW == 1) {
				total = __shfl_sync(0xffffffffu, wi, 31);
			} else {
				if (lane == 31) sh.wsum[wid] = wi;
				if (t == 0) sh.first = NT;
				group_sync<NT>(bar);
				total = 0.0;
#pragma unroll
				for (int k = 0; k < NW; k++) {
					const double v = sh.wsum[k];
					if (k < wid) woff += v;
					total += v;
				}
			}
			double TMj = 0.0, absorb = 0.0, TMafter = 0.0;
			bool capped = false, cut = false;
			double a0 = 0.0, a1 = 0.0, a2 = 0.0;
			if (part) {
				const double excl = (woff + wi) - my_tau;
				TMj = TM * exp(-excl);
				absorb = TMj * -expm1(-my_tau);
				TMafter = TMj - absorb;
				a0 = t0 / my_tau * absorb;
				capped = a0 > NHI;
				if (he) {
					a1 = t1 / my_tau * absorb;
					a2 = t2 / my_tau * absorb;
					capped = capped || a1 > N1 || a2 > N2;
				}
				cut = below_cutoff(TMafter, Nph);
			}
			int f;
			if (NW == 1) {
				const unsigned ev = __ballot_sync(0xffffffffu, capped || cut);
				f = ev ? __ffs(ev) - 1 : NT;
			} else {
				if (capped || cut) atomicMin(&sh.first, t);
				group_sync<NT>(bar);
				f = sh.first;
			}
			if (part && t < f) {
				d0 = a0 * NH_inv;
				if (he) { d1 = a1 * NHe_inv; d2 = a2 * NHe_inv; }
				delta = d0;
			}
			if (f == NT) {
				TM = TM * exp(-total);
				group_sync<NT>(bar);       // shared words are rewritten by the next step
				break;
			}
			double TMnew = 0.0;
			if (t == f) {
				TMnew = TMafter;
				if (capped) {
					if (a0 > NHI) { a0 = NHI; nsat++; }
					double ab = a0;
					if (he) {
						if (a1 > N1) { a1 = N1; nsat++; }
						if (a2 > N2) { a2 = N2; nsat++; }
						ab += (a1 + a2);
					}
					TMnew = TMj - ab;
				}
				d0 = a0 * NH_inv;
				if (he) { d1 = a1 * NHe_inv; d2 = a2 * NHe_inv; }
				delta = d0;
				if (NW > 1) sh.tm = TMnew;
			}
			if (NW == 1) {
				TM = __shfl_sync(0xffffffffu, TMnew, f);
			} else {
				group_sync<NT>(bar);
				TM = sh.tm;
			}
			if (below_cutoff(TM, Nph)) done = true;
			start = f + 1;
			group_sync<NT>(bar);
		}
		if (valid) {
			// loop.c:512-552: yGdep increments and heat of the hit
			double y0 = delta, y1 = 0.0, y2 = 0.0, heat = 0.0;
			if (delta >= 0.0) {
				if (P.secondary && xe > 0.0) {
					const double lx = log10(xe);
					y0 = d0 + (d0 * dE0 / P.HI_ENERGY * secion_get(P, 0, dE0, lx) +
							d1 * dE1 / P.HI_ENERGY * secion_get(P, 0, dE1, lx));
					heat = hf0 * d0 * secion_get(P, 2, dE0, lx);
					if (he) {
						y1 = d1 + (d0 * dE0 / P.HEI_ENERGY * secion_get(P, 1, dE0, lx) +
								d1 * dE1 / P.HEI_ENERGY * secion_get(P, 1, dE1, lx));
						heat += hf1 * d1 * secion_get(P, 2, dE1, lx);
						y2 = d2;
					}
				} else {
					heat = hf0 * d0;
					if (he) {
						y1 = d1;
						y2 = d2;
						heat += d1 * hf1;
						heat += d2 * hf2;
					}
				}
			}
			acc_store(acc, nacc, slot_c, y0, heat, y1, y2);
		}
	}
	if (t == 0 && !skip_ray) lost += TM;
}

// A tick's rays by deposit group: long rays (a whole block each), middle
// rays (a 128-thread quarter each) and short rays (a warp each), as ranges
// of the batch's three ray lists. Filled on the device (k_tick_rays).
struct TickRays {
	int l0, nlong, m0, nmid, s0, nshort, pad0, pad1;
};

// Work units of a tick: [0, nlong) take one long ray each with all
// DEP_THREADS threads; the next ceil(nmid/4) take four middle rays each, 128
// threads per ray; the rest take DEP_THREADS/32 short rays, one per warp.
// The grid is persistent: blocks claim units from the tick's counter, so
// the launch needs no count from the host.
#define DEP_THREADS 512
#define DEP_LONG 96       // more hits than this: a group of threads, else a warp
#define DEP_MID 384       // more hits than this: the whole block, else a 128-thread quarter

template <bool GEN, bool AFF>
__global__ void __launch_bounds__(DEP_THREADS, 2) k_deposit(int t, const TickRays *__restrict__ tick_rays,
		unsigned *__restrict__ unit_ctr, const PsgBatchDev *__restrict__ B,
		const uint32_t *__restrict__ long_rays, const uint32_t *__restrict__ mid_rays,
		const uint32_t *__restrict__ short_rays,
		const int64_t *__restrict__ off, const uint32_t *__restrict__ hipar, const double *__restrict__ hkern,
		const double *__restrict__ lambdaH, const float *__restrict__ mass,
		PhysParams P, int want_heat, double *__restrict__ acc, int nacc, unsigned long long *__restrict__ n_sat,
		double *__restrict__ lost) {
	__shared__ DepShared sh_block;
	__shared__ DepShared sh_quarter[4];
	__shared__ DepShared sh_warp[DEP_THREADS / 32];
	__shared__ int s_unit;
	const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
	unsigned nsat = 0;
	double tm_lost = 0.0;
	const psg_ray *__restrict__ rays = B->rays;      // read here: a replayed graph serves any call's rays
	const TickRays T = tick_rays[t];
	const int nlong = T.nlong, nmid = T.nmid, nshort = T.nshort;
	const int nmid_blocks = (nmid + 3) / 4;
	const int nunits = nlong + nmid_blocks + (nshort + DEP_THREADS / 32 - 1) / (DEP_THREADS / 32);
	for (;;) {
		if (tid == 0) s_unit = (int)atomicAdd(unit_ctr + t, 1u);
		__syncthreads();
		const int u = s_unit;
		__syncthreads();       // (also: the previous unit's shared state is no longer read)
		if (u >= nunits) break;
		if (u < nlong) {
			const uint32_t r = long_rays[T.l0 + u];
			if (GEN)
				deposit_ray_gen<DEP_THREADS>(rays[r], off[r], off[r + 1], tid, hipar, hkern, lambdaH, mass, P,
						want_heat, acc, nacc, sh_block, nsat, tm_lost, 0);
			else
				deposit_ray<DEP_THREADS, AFF>(rays[r], off[r], off[r + 1], tid, hipar, hkern, lambdaH, mass, P,
						want_heat, acc, sh_block, nsat, tm_lost, 0);
		} else if (u < nlong + nmid_blocks) {
			const int q = tid >> 7;
			const int m = (u - nlong) * 4 + q;
			if (m < nmid) {
				const uint32_t r = mid_rays[T.m0 + m];
				if (GEN)
					deposit_ray_gen<128>(rays[r], off[r], off[r + 1], tid & 127, hipar, hkern, lambdaH, mass, P,
							want_heat, acc, nacc, sh_quarter[q], nsat, tm_lost, 1 + q);
				else
					deposit_ray<128, AFF>(rays[r], off[r], off[r + 1], tid & 127, hipar, hkern, lambdaH, mass, P,
							want_heat, acc, sh_quarter[q], nsat, tm_lost, 1 + q);
			}
		} else {
			const int w = (u - nlong - nmid_blocks) * (DEP_THREADS / 32) + wid;
			if (w < nshort) {
				const uint32_t r = short_rays[T.s0 + w];
				if (off[r + 1] > off[r]) {
					if (GEN)
						deposit_ray_gen<32>(rays[r], off[r], off[r + 1], lane, hipar, hkern, lambdaH, mass, P,
								want_heat, acc, nacc, sh_warp[wid], nsat, tm_lost, 0);
					else
						deposit_ray<32, AFF>(rays[r], off[r], off[r + 1], lane, hipar, hkern, lambdaH, mass, P,
								want_heat, acc, sh_warp[wid], nsat, tm_lost, 0);
				}
			}
		}
	}
	for (int o = 16; o > 0; o >>= 1) nsat += __shfl_down_sync(0xffffffffu, nsat, o);
	if (lane == 0 && nsat) atomicAdd(n_sat, (unsigned long long)nsat);
	if (lane == 0 && tm_lost != 0.0) atomicAdd(lost, tm_lost);
}

// Per tick, the ranges of its rays in the long / middle / short lists, from
// the classes' running counts (the lists keep ray order, so each tick's rays
// are a run of each list).
__global__ void k_tick_rays(int K, size_t R, size_t nray, const unsigned long long *__restrict__ cls,
		const unsigned long long *__restrict__ scan, TickRays *__restrict__ out) {
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= K) return;
	const unsigned long long tot = scan[nray - 1] + cls[nray - 1];
	const unsigned long long c0 = scan[(size_t)t * R], c1 = (t + 1 < K) ? scan[(size_t)(t + 1) * R] : tot;
	TickRays T;
	T.l0 = (int)(uint32_t)c0;
	T.m0 = (int)(uint32_t)(c0 >> 32);
	T.nlong = (int)(uint32_t)c1 - T.l0;
	T.nmid = (int)(uint32_t)(c1 >> 32) - T.m0;
	T.s0 = (int)((size_t)t * R) - T.l0 - T.m0;
	T.nshort = (int)R - T.nlong - T.nmid;
	T.pad0 = T.pad1 = 0;
	out[t] = T;
}

// Rays of the batch split into long, middle and short lists (ray order
// kept): cls = 1 for long, 1 << 32 for middle, so one scan counts both.
// (dep_long and dep_mid: the thresholds, DEP_LONG and DEP_MID unless tuned)
__global__ void k_ray_class(size_t nray, const int64_t *__restrict__ off, int dep_long, int dep_mid,
		unsigned long long *__restrict__ cls) {
	const size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
	if (r >= nray) return;
	const int64_t n = off[r + 1] - off[r];
	cls[r] = n > dep_mid ? 1ull : (n > dep_long ? (1ull << 32) : 0ull);
}

// (each list has room for every ray of the batch)
__global__ void k_ray_lists(size_t nray, const unsigned long long *__restrict__ cls,
		const unsigned long long *__restrict__ scan, uint32_t *__restrict__ long_rays,
		uint32_t *__restrict__ mid_rays, uint32_t *__restrict__ short_rays) {
	const size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
	if (r >= nray) return;
	const unsigned long long sc = scan[r];
	const uint32_t nl = (uint32_t)sc, nm = (uint32_t)(sc >> 32);
	if (cls[r] == 1ull) long_rays[nl] = (uint32_t)r;
	else if (cls[r]) mid_rays[nm] = (uint32_t)r;
	else short_rays[r - nl - nm] = (uint32_t)r;
}

// Active particles of the batch whose deposit segment is longer than a warp
// (particles next to a source are hit by nearly every ray); flag[na] = 0 so
// that the scan's last entry is the total.
// The active count of the batch, nact = tick_act[K], is read on the device;
// flags cover the capacity cap + 1 (zero past nact) so the scan's size is
// fixed.
// The active pairs whose run is longer than short_max hits, per tick (their order
// within a tick is free: each is summed and sorted on its own). Counted per
// tick, the K counts scanned by one block, then listed; runs longer than
// SLOT_WARP_MAX also go to the lists of the two block sorts.
__device__ __forceinline__ int tick_of_pair(const int32_t *__restrict__ tick_act, int K, int a) {
	int lo = 0, hi = K;      // last t with tick_act[t] <= a
	while (hi - lo > 1) {
		const int mid = (lo + hi) >> 1;
		if (tick_act[mid] <= a) lo = mid;
		else hi = mid;
	}
	return lo;
}
// (a warp's pairs are consecutive and mostly of one tick: one atomic per
// tick per warp, the lanes ranked within it)
__global__ void k_long_count(const int32_t *__restrict__ tick_act, int K, const uint32_t *__restrict__ act_seg,
		uint32_t short_max, unsigned long long *__restrict__ tick_cnt) {
	const int na = tick_act[K];
	const int lane = threadIdx.x & 31;
	const int stride = (int)(gridDim.x * blockDim.x);
	for (int a0 = (int)(blockIdx.x * blockDim.x + threadIdx.x) - lane; a0 < na; a0 += stride) {
		const int a = a0 + lane;
		const bool is_long = a < na && act_seg[a + 1] - act_seg[a] > short_max;
		const int t = is_long ? tick_of_pair(tick_act, K, a) : -1;
		const unsigned grp = __match_any_sync(0xffffffffu, t);
		if (is_long && lane == __ffs(grp) - 1) atomicAdd(&tick_cnt[t], (unsigned long long)__popc(grp));
	}
}
__global__ void k_long_place(const int32_t *__restrict__ tick_act, int K, const uint32_t *__restrict__ act_seg,
		uint32_t short_max, const unsigned long long *__restrict__ tick_off, unsigned *__restrict__ cursor,
		uint32_t *__restrict__ long_act, int32_t *__restrict__ tick_long, uint32_t *__restrict__ mid_list,
		unsigned *__restrict__ mid_count, uint32_t *__restrict__ vl_list, unsigned *__restrict__ vl_count) {
	const int na = tick_act[K];
	const int lane = threadIdx.x & 31;
	const int i0 = (int)(blockIdx.x * blockDim.x + threadIdx.x);
	const int stride = (int)(gridDim.x * blockDim.x);
	for (int t = i0; t <= K; t += stride) tick_long[t] = (int32_t)tick_off[t];
	for (int a0 = i0 - lane; a0 < na; a0 += stride) {
		const int a = a0 + lane;
		const uint32_t n = a < na ? act_seg[a + 1] - act_seg[a] : 0u;
		const bool is_long = n > short_max;
		const int t = is_long ? tick_of_pair(tick_act, K, a) : -1;
		const unsigned grp = __match_any_sync(0xffffffffu, t);
		const int leader = __ffs(grp) - 1;
		unsigned base = 0;
		if (is_long && lane == leader) base = atomicAdd(&cursor[t], (unsigned)__popc(grp));
		base = __shfl_sync(0xffffffffu, base, leader);
		if (!is_long) continue;
		long_act[tick_off[t] + base + __popc(grp & ((1u << lane) - 1u))] = (uint32_t)a;
		if (n > SLOT_MID_MAX) vl_list[atomicAdd(vl_count, 1u)] = (uint32_t)a;
		else if (n > SLOT_WARP_MAX) mid_list[atomicAdd(mid_count, 1u)] = (uint32_t)a;
	}
}

// One active particle's non-isothermal update, prepared by k_reduce<false>
// so that the integrator reads one contiguous record instead of gathering
// the particle's state: the inputs of the step and f(x0) (with the
// recombination photons' rate when not on the spot). 80 bytes, a multiple
// of 16 for cp.async.
struct __align__(16) UpdRec {
	double time, lam0, g, heat, k0, k1;
	float ie0, rho, yeMET, hstep;
	uint32_t p, pad0;
	double krec;
};
static_assert(sizeof(UpdRec) == 80, "UpdRec layout");

// An integration that looks long (the integrator queue claims these first):
// no step proposal carried over, a proposal under a quarter of the step, or
// more photons absorbed than the particle has neutral atoms.
__device__ __forceinline__ bool upd_looks_slow(float hstep, double time, double g, double lam0) {
	return !(hstep > 0.0f) || 4.0 * (double)hstep < time || g > lam0;
}

// The particle's summed deposits of the tick: isothermal, the closed-form
// update_pars() step (loop.c:653-770); otherwise the sums for the integrator
// (with act_slow, whether the integrator should claim it first).
template <bool ISO, bool REC>
__device__ __forceinline__ void finish_particle(int a, double g, double heat, int nh,
		const uint32_t *__restrict__ act_ipar, int32_t *__restrict__ hits, double *__restrict__ act_g,
		double *__restrict__ act_heat, double *__restrict__ lambdaH, float *__restrict__ ie,
		int64_t *__restrict__ lasthit, const float *__restrict__ rho, const float *__restrict__ yeMET,
		const float *__restrict__ hstep, UpdRec *__restrict__ rec, int lo, const double *__restrict__ gcarry,
		uint8_t *__restrict__ act_slow, const PhysParams &P, int64_t tick, double tick_time,
		uint32_t *__restrict__ status) {
	const uint32_t p = act_ipar[a];
	hits[p] += nh;
	if (gcarry) g += gcarry[p];      // photons left over by an earlier explicit step (loop.c:745)
	if (!ISO) {
		if (act_g) {        // read by the integrator queue, the surrogate and the update log
			act_g[a] = g;
			act_heat[a] = heat;
		}
		if (act_slow)
			act_slow[a] = upd_looks_slow(hstep[p], rn_dmul((double)(tick - lasthit[p]), tick_time), g, lambdaH[p]);
		if (!rec) return;      // sums only: the integrator builds its own records
		UpdRec r;
		r.time = rn_dmul((double)(tick - lasthit[p]), tick_time);
		r.lam0 = lambdaH[p];
		r.g = g;
		r.heat = heat;
		r.ie0 = ie[p];
		r.rho = rho[p];
		r.yeMET = yeMET[p];
		r.hstep = hstep[p];
		r.p = p;
		r.pad0 = 0u;
		r.krec = 0.0;
		const double ie0 = (double)r.ie0;
		const double T = ieye2T(P, ie0, rn_dadd(rn_dsub(1.0, r.lam0), P.he_e));
		const RhsCtx cx = make_rhs_ctx(P, (double)r.yeMET, g, heat, r.time, rn_dmul(P.H_PER_MASS, (double)r.rho), T);
		const double x0[2] = {r.lam0, ie0};
		double f0[2];
		rhs<REC, true>(P, cx, x0, f0, &r.krec);
		r.k0 = f0[0];
		r.k1 = f0[1];
		rec[a - lo] = r;    // records of one tick, from its first active particle
		return;
	}
	const double time = rn_dmul((double)(tick - lasthit[p]), tick_time);
	const double lam0 = lambdaH[p];
	const double T = ieye2T(P, (double)ie[p], rn_dadd(rn_dsub(1.0, lam0), P.he_e));
	const double nH = rn_dmul(P.H_PER_MASS, (double)rho[p]);
	double lam = lam0, grec = 0.0;
	const uint32_t st = solve_step_iso(P, lam, (double)yeMET[p], g, time, nH, T, REC ? &grec : nullptr);
	lambdaH[p] = lam;
	if (REC) P.ygrec[p] = (float)fmax(0.0, (double)P.ygrec[p] + grec);     // x[3], solve.c:183,211,218
	ie[p] = (float)Tye2ie(P, T, rn_dadd(rn_dsub(1.0, lam), P.he_e));
	lasthit[p] = tick;
	if (st) atomicOr(status, st);
}

// Runs of up to short_max (at most RUN_SHORT) hits stay in placement order; their
// sums go in hit order all the same. Up to 4 hits by selection (each step
// the smallest hit index above the last: at most 16 reads, in L1); up to 8
// and 16 through a bitonic network in registers (fully unrolled: 24 and 80
// compare-exchanges). Longer runs are sorted and read in order.
__device__ __forceinline__ uint32_t next_in_run(const uint32_t *__restrict__ vals, uint32_t s0, uint32_t s1,
		int64_t prev) {
	uint32_t best = 0xFFFFFFFFu;
	for (uint32_t q = s0; q < s1; q++) {
		const uint32_t v = vals[q];
		if ((int64_t)v > prev && v < best) best = v;
	}
	return best;
}
template <int N>
__device__ __forceinline__ void bitonic_regs(uint32_t (&v)[N]) {
#pragma unroll
	for (int k = 2; k <= N; k <<= 1) {
#pragma unroll
		for (int j = k >> 1; j > 0; j >>= 1) {
#pragma unroll
			for (int i = 0; i < N; i++) {
				const int l = i ^ j;
				if (l > i) {
					const uint32_t a = v[i], b = v[l];
					const bool up = (i & k) == 0;
					v[i] = up ? min(a, b) : max(a, b);
					v[l] = up ? max(a, b) : min(a, b);
				}
			}
		}
	}
}
template <int N, typename F>
__device__ __forceinline__ void visit_sorted_regs(const uint32_t *__restrict__ vals, uint32_t s0, uint32_t n, F f) {
	uint32_t v[N];
#pragma unroll
	for (int i = 0; i < N; i++) v[i] = (uint32_t)i < n ? vals[s0 + i] : 0xFFFFFFFFu;
	bitonic_regs<N>(v);
#pragma unroll
	for (int i = 0; i < N; i++)
		if ((uint32_t)i < n) f(v[i]);
}
// f(hit) for every hit of the run [s0, s1) in hit order; runs longer than
// short_max (4, 8 or 16: the tuner's run_short) are read as stored (sorted)
template <typename F>
__device__ __forceinline__ void visit_run(const uint32_t *__restrict__ vals, uint32_t s0, uint32_t s1,
		uint32_t short_max, F f) {
	const uint32_t n = s1 - s0;
	if (n > short_max) {
		for (uint32_t k = s0; k < s1; k++) f(vals[k]);
	} else if (n <= 4) {
		int64_t prev = -1;
		for (uint32_t i = 0; i < n; i++) {
			const uint32_t h = next_in_run(vals, s0, s1, prev);
			prev = h;
			f(h);
		}
	} else if (n <= 8) {
		visit_sorted_regs<8>(vals, s0, n, f);
	} else {
		visit_sorted_regs<RUN_SHORT>(vals, s0, n, f);
	}
}

// One long deposit segment [b0, b1) summed by a warp: lanes strided over
// it (eight loads in flight per lane), then a fixed butterfly; every lane
// ends with the totals. Slot k's deposits sit at hit vals[k].
__device__ __forceinline__ void warp_segment_sum(const double *__restrict__ acc, const uint32_t *__restrict__ vals,
		int want_heat, uint32_t b0, uint32_t b1, int lane, double &sg, double &sh, int &sn) {
	sg = 0.0;
	sh = 0.0;
	sn = 0;
	uint32_t k = b0 + lane;
	if (want_heat) {
		const double2 *acc2 = reinterpret_cast<const double2 *>(acc);
		for (; k + 7 * 32 < b1; k += 8 * 32) {
			uint32_t hv[8];
			double2 v[8];
#pragma unroll
			for (int u = 0; u < 8; u++) hv[u] = vals[k + 32 * u];
#pragma unroll
			for (int u = 0; u < 8; u++) v[u] = acc2[hv[u]];
#pragma unroll
			for (int u = 0; u < 8; u++)
				if (v[u].x >= 0.0) { sg += v[u].x; sh += v[u].y; sn++; }
		}
		for (; k < b1; k += 32) {
			const double2 d = acc2[vals[k]];
			if (d.x >= 0.0) { sg += d.x; sh += d.y; sn++; }
		}
	} else {
		for (; k + 7 * 32 < b1; k += 8 * 32) {
			uint32_t hv[8];
			double v[8];
#pragma unroll
			for (int u = 0; u < 8; u++) hv[u] = vals[k + 32 * u];
#pragma unroll
			for (int u = 0; u < 8; u++) v[u] = acc[hv[u]];
#pragma unroll
			for (int u = 0; u < 8; u++)
				if (v[u] >= 0.0) { sg += v[u]; sn++; }
		}
		for (; k < b1; k += 32) {
			const double d = acc[vals[k]];
			if (d >= 0.0) { sg += d; sn++; }
		}
	}
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) {
		sg += __shfl_xor_sync(0xffffffffu, sg, o);
		sh += __shfl_xor_sync(0xffffffffu, sh, o);
		sn += __shfl_xor_sync(0xffffffffu, sn, o);
	}
}

// Per-particle sums of one tick's deposits (photons/NH, heat, deposit count)
// in hit order. Warps first take the tick's segments of more than RUN_THREAD
// deposits, a warp each (particles are in leaf order, so the long ones are
// neighbours; giving each its own warp keeps them from piling up on a few
// warps), then every thread takes shorter ones, a thread each (sorted runs
// read in order, shorter ones put in hit order by visit_run). The grid is
// persistent (both loops stride over the tick's ranges, read on the device).
template <bool ISO, bool REC>
__global__ void __launch_bounds__(256) k_reduce(int t, const int32_t *__restrict__ tick_act,
		const uint32_t *__restrict__ act_ipar, const uint32_t *__restrict__ act_seg,
		const double *__restrict__ acc, const uint32_t *__restrict__ vals, uint32_t short_max, int want_heat,
		const uint32_t *__restrict__ long_act, const int32_t *__restrict__ tick_long,
		int32_t *__restrict__ hits, double *__restrict__ act_g, double *__restrict__ act_heat,
		double *__restrict__ lambdaH, float *__restrict__ ie, int64_t *__restrict__ lasthit,
		const float *__restrict__ rho, const float *__restrict__ yeMET, const float *__restrict__ hstep,
		UpdRec *__restrict__ rec, const double *__restrict__ gcarry, uint8_t *__restrict__ act_slow, PhysParams P,
		const PsgBatchDev *__restrict__ B, uint32_t *__restrict__ status) {
	const int64_t tick = B->tick0 + t;
	const double tick_time = B->tick_time;
	const int lo = tick_act[t], hi = tick_act[t + 1];
	const int lane = threadIdx.x & 31;
	const int nwarp = (int)((gridDim.x * blockDim.x) >> 5);
	for (int e = tick_long[t] + (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); e < tick_long[t + 1];
			e += nwarp) {
		const int a = (int)long_act[e];
		if (act_seg[a + 1] - act_seg[a] <= RUN_THREAD) continue;      // (a thread's, below)
		double sg, sh;
		int sn;
		warp_segment_sum(acc, vals, want_heat, act_seg[a], act_seg[a + 1], lane, sg, sh, sn);
		if (lane == 0)
			finish_particle<ISO, REC>(a, sg, sh, sn, act_ipar, hits, act_g, act_heat, lambdaH, ie, lasthit, rho, yeMET,
					hstep, rec, lo, gcarry, act_slow, P, tick, tick_time, status);
	}
	for (int a = lo + (int)(blockIdx.x * blockDim.x + threadIdx.x); a < hi; a += (int)(gridDim.x * blockDim.x)) {
		const uint32_t s0 = act_seg[a], s1 = act_seg[a + 1];
		if (s1 - s0 > RUN_THREAD) continue;
		double g = 0.0, heat = 0.0;
		int nh = 0;
		visit_run(vals, s0, s1, short_max, [&](uint32_t hk) {
			if (want_heat) {
				const double2 d = reinterpret_cast<const double2 *>(acc)[hk];
				if (d.x >= 0.0) { g += d.x; heat += d.y; nh++; }
			} else {
				const double d = acc[hk];
				if (d >= 0.0) { g += d; nh++; }
			}
		});
		finish_particle<ISO, REC>(a, g, heat, nh, act_ipar, hits, act_g, act_heat, lambdaH, ie, lasthit, rho, yeMET,
				hstep, rec, lo, gcarry, act_slow, P, tick, tick_time, status);
	}
}

// update_pars() loop.c:653-770, not isothermal: every lane integrates one
// particle at a time with the Dormand-Prince step; a lane whose particle is
// done takes the next one of the tick from a shared cursor, so the warp keeps
// all lanes on integrator steps (particles need 1 to a few hundred steps).
#define UPD_MAX_STEPS 200000
struct StiffItem {
	double t, h, x0, x1, yeMET, g, heat, time, nH, T, rec;
	uint32_t p;
};
#define UPD_WARPS 8
// Where the integrator's records come from: the tick's active particles,
// their summed deposits (act_g, act_heat, from k_reduce) and the particle
// state.
struct UpdSrc {
	const uint32_t *act_ipar;
	const double *act_g, *act_heat;
	const float *rho, *yeMET;
	const uint8_t *slow;      // per active pair: claim in the first pass (with cursor2)
};

// Every warp owns two buffers of 32 records in shared memory: it claims
// chunks of 32 particles from the tick's cursor and builds their records
// (the summed deposits, the state, the step length) one chunk ahead, so a
// lane whose particle is done takes the next one from shared memory; the
// gathers of a chunk are paid once per 32 particles, not per integrator
// step, and no record goes through device memory. MINB caps the registers
// for that many resident blocks per multiprocessor (psg_tune).
//
// With cursor2 (psg_tune.update_order) the tick's particles are claimed in
// two passes: first, from cursor, those that look slow (src.slow, set by
// k_reduce before this kernel starts, so both passes see the same flags:
// no step proposal carried over -- new, or handed to the stiff finish last
// time --, a proposal under a quarter of this step, or more photons absorbed
// than neutral atoms), then, from cursor2, the others; each claim keeps its
// chunk's particles of the pass. Long integrations then start early instead
// of trailing the kernel on a few lanes. Which lane integrates a particle
// changes, not its result.
template <bool REC, int MINB>
__global__ void __launch_bounds__(32 * UPD_WARPS, MINB) k_update_queue(int t, const int32_t *__restrict__ tick_act,
		const UpdSrc src, double *__restrict__ lambdaH, float *__restrict__ ie,
		int64_t *__restrict__ lasthit, float *__restrict__ hstep, PhysParams P, const PsgBatchDev *__restrict__ B,
		unsigned *__restrict__ cursor, unsigned *__restrict__ cursor2, StiffItem *__restrict__ stiff,
		unsigned *__restrict__ nstiff, const uint32_t *__restrict__ alist, const unsigned *__restrict__ nalist,
		uint32_t *__restrict__ status) {
	__shared__ UpdRec buf[UPD_WARPS][2][32];
	const int64_t tick = B->tick0 + t;
	const double tick_time = B->tick_time;
	// the tick's particles, or only those listed in alist (the surrogate's rejects)
	const int lo = tick_act[t], hi = tick_act[t + 1];
	const unsigned n = alist ? *nalist : (unsigned)(hi - lo);
	const int lane = threadIdx.x & 31;
	const unsigned lt_mask = (1u << lane) - 1u;
	UpdRec (*WB)[32] = buf[threadIdx.x >> 5];
	int pass = 0;        // warp-uniform: 0 the slow-looking particles (or all), 1 the others
	// fills WB[b] with the next particles of the pass, packed from slot 0;
	// returns how many (0: none left)
	auto fetch = [&](int b) -> int {
		for (;;) {
			unsigned base = 0;
			if (lane == 0) base = atomicAdd(pass ? cursor2 : cursor, 32u);
			base = __shfl_sync(0xffffffffu, base, 0);
			if (base >= n) {
				if (cursor2 && pass == 0) {
					pass = 1;
					continue;
				}
				return 0;
			}
			const int cnt = (int)min(32u, n - base);
			bool keep = false;
			UpdRec r;
			if (lane < cnt) {
				const unsigned k = base + lane;
				const int a = alist ? (int)alist[k] : lo + (int)k;
				keep = !cursor2 || (src.slow[a] != 0) == (pass == 0);
				if (keep) {
					const uint32_t p = src.act_ipar[a];
					r.time = rn_dmul((double)(tick - lasthit[p]), tick_time);
					r.lam0 = lambdaH[p];
					r.g = src.act_g[a];
					r.heat = src.act_heat[a];
					r.ie0 = ie[p];
					r.rho = src.rho[p];
					r.yeMET = src.yeMET[p];
					r.hstep = hstep[p];
					r.p = p;
					r.pad0 = 0u;
					r.k0 = r.k1 = r.krec = 0.0;
				}
			}
			const unsigned km = __ballot_sync(0xffffffffu, keep);
			if (keep) WB[b][__popc(km & lt_mask)] = r;
			__syncwarp();
			if (km) return __popc(km);
		}
	};
	int avail[2];
	avail[0] = fetch(0);
	avail[1] = fetch(1);
	int cur = 0, used = 0;
	bool exhausted = false;
	DPState S;
	RhsCtx cx;
	double atol1 = 0.0;
	uint32_t p = 0;
	bool have = false;
	uint32_t st = 0;
	for (;;) {
		unsigned need = __ballot_sync(0xffffffffu, !have);
		while (need && !exhausted) {
			const int left = avail[cur] - used;
			if (left <= 0) {
				if (avail[cur ^ 1] == 0) {
					exhausted = true;
					break;
				}
				cur ^= 1;
				used = 0;
				avail[cur ^ 1] = fetch(cur ^ 1);
				continue;
			}
			const int rank = __popc(need & lt_mask);
			const int take = min(__popc(need), left);
			if (!have && rank < take) {
				const UpdRec &r = WB[cur][used + rank];
				p = r.p;
				const double ie0 = (double)r.ie0;
				const double T = ieye2T(P, ie0, rn_dadd(rn_dsub(1.0, r.lam0), P.he_e));
				cx = make_rhs_ctx(P, (double)r.yeMET, r.g, r.heat, r.time, rn_dmul(P.H_PER_MASS, (double)r.rho), T);
				S.x[0] = r.lam0;
				S.x[1] = ie0;
				S.rec = 0.0;
				rhs<REC, true>(P, cx, S.x, S.k1, &S.krec);
				atol1 = DP_ATOL1_REL * fabs(ie0) + 1e-300;
				dp_init_k1(S);
				// the particle's last step proposal is a better first
				// step than the derivative estimate
				if (r.hstep > 0.0f) S.h = fmin(1.0, fmax((double)r.hstep / r.time, 1e-8));
				have = true;
			}
			used += take;
			need = __ballot_sync(0xffffffffu, !have);
		}
		if (!__any_sync(0xffffffffu, have)) break;
		if (have) {
			const bool done = dp_step<REC>(P, cx, S, atol1);
			if (!done && S.steps >= DP_SWITCH) {
				// stiff: hand the particle to k_update_stiff and free the lane
				const unsigned q = atomicAdd(nstiff, 1u);
				StiffItem it;
				it.p = p; it.t = S.t; it.h = S.h; it.x0 = S.x[0]; it.x1 = S.x[1];
				it.yeMET = cx.yeMET; it.g = cx.g; it.heat = cx.heat; it.time = cx.time; it.nH = cx.nH; it.T = cx.T;
				it.rec = S.rec;
				stiff[q] = it;
				hstep[p] = 0.0f;
				have = false;
			} else if (done) {
				const double lam = S.x[0], e = S.x[1];
				if (!(e >= 0.0)) st |= PSG_ST_IE_NEG;
				if (!isfinite(lam) || !isfinite(e)) st |= PSG_ST_NAN;
				lambdaH[p] = fmin(1.0, fmax(0.0, lam));
				if (!P.adiabatic) ie[p] = (float)e;
				if (REC) P.ygrec[p] = (float)fmax(0.0, (double)P.ygrec[p] + S.rec);
				lasthit[p] = tick;
				hstep[p] = (float)((double)S.hnext * cx.time);
				have = false;
			}
		}
	}
	if (st) atomicOr(status, st);
}

// The stiff particles of a tick, one thread each (their number is read on
// the device): Rosenbrock from where the explicit steps stopped.
template <bool REC>
__global__ void __launch_bounds__(64) k_update_stiff(const StiffItem *__restrict__ stiff,
		const unsigned *__restrict__ nstiff, double *__restrict__ lambdaH, float *__restrict__ ie,
		int64_t *__restrict__ lasthit, PhysParams P, const PsgBatchDev *__restrict__ B, int t,
		uint32_t *__restrict__ status) {
	const int64_t tick = B->tick0 + t;
	const unsigned n = *nstiff;
	uint32_t st = 0;
	for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
		const StiffItem it = stiff[i];
		const RhsCtx cx = make_rhs_ctx(P, it.yeMET, it.g, it.heat, it.time, it.nH, it.T);
		double x[2] = {it.x0, it.x1};
		double rec = it.rec;
		if (!rosenbrock<REC>(P, cx, x, it.t, it.h, UPD_MAX_STEPS, &rec)) st |= PSG_ST_SOLVER;
		if (REC) P.ygrec[it.p] = (float)fmax(0.0, (double)P.ygrec[it.p] + rec);
		if (!(x[1] >= 0.0)) st |= PSG_ST_IE_NEG;
		if (!isfinite(x[0]) || !isfinite(x[1])) st |= PSG_ST_NAN;
		lambdaH[it.p] = fmin(1.0, fmax(0.0, x[0]));
		if (!P.adiabatic) ie[it.p] = (float)x[1];
		lasthit[it.p] = tick;
	}
	if (st) atomicOr(status, st);
}

// update_pars() with step_evolve_euler(): one thread per active particle
// from its record; the unused fraction of the absorbed photons is carried
// to the particle's next update (loop.c:745), heat is not (loop.c:769).
__global__ void __launch_bounds__(128) k_update_euler(int t, const int32_t *__restrict__ tick_act,
		const UpdRec *__restrict__ rec, double *__restrict__ lambdaH, float *__restrict__ ie,
		int64_t *__restrict__ lasthit, double *__restrict__ gcarry, PhysParams P, const PsgBatchDev *__restrict__ B,
		uint32_t *__restrict__ status) {
	const int64_t tick = B->tick0 + t;
	const int lo = tick_act[t], hi = tick_act[t + 1];
	for (int a = lo + (int)(blockIdx.x * blockDim.x + threadIdx.x); a < hi; a += (int)(gridDim.x * blockDim.x)) {
	const UpdRec r = rec[a - lo];
	const double ie0 = (double)r.ie0;
	const double T = ieye2T(P, ie0, rn_dadd(rn_dsub(1.0, r.lam0), P.he_e));
	const RhsCtx cx = make_rhs_ctx(P, (double)r.yeMET, r.g, r.heat, r.time, rn_dmul(P.H_PER_MASS, (double)r.rho), T);
	double x[2] = {r.lam0, ie0};
	double remain = 0.0, grec = 0.0;
	int refined = 0;
	uint32_t st = P.ygrec ? euler_step<true>(P, cx, x, remain, refined, &grec) : euler_step<false>(P, cx, x, remain, refined);
	if (P.ygrec) P.ygrec[r.p] = (float)((double)P.ygrec[r.p] + grec);
	const double lam = fmin(1.0, fmax(0.0, x[0]));
	lambdaH[r.p] = lam;
	if (P.isothermal) ie[r.p] = (float)Tye2ie(P, T, rn_dadd(rn_dsub(1.0, lam), P.he_e));
	else if (!P.adiabatic) ie[r.p] = (float)x[1];
	lasthit[r.p] = tick;
	gcarry[r.p] = r.g * remain;
	if (st) atomicOr(status, st);
	}
}

// update_pars() loop.c:647-776 with helium: one thread per active particle
// of the tick sums its deposits (yGdepHI, heat, yGdepHeI, yGdepHeII, in slot
// order) and integrates the four variables; isothermal, ie follows T at the
// new ye (loop.c:764-766). A particle still unfinished after the explicit
// steps goes to k_update_he_stiff (the Rosenbrock finish), which keeps the
// W-method's registers out of this kernel.
struct HeStiffItem {
	HeStep s;
	double x[4], rec[3], t, h;
	uint32_t p;
};

// The step's results into the particle (update_pars() loop.c:756-768).
__device__ __forceinline__ void he_write(const PhysParams &P, uint32_t p, const double x[4], const double rec[3],
		double T, int64_t tick, double *__restrict__ lambdaH, float *__restrict__ ie, int64_t *__restrict__ lasthit) {
	lambdaH[p] = x[0];
	P.lamHeI[p] = x[1];
	P.lamHeII[p] = x[2];
	if (P.ygrec) {
		P.ygrec[p] = (float)rec[0];
		P.ygrecHe1[p] = (float)rec[1];
		P.ygrecHe2[p] = (float)rec[2];
	}
	if (P.isothermal) ie[p] = (float)Tye2ie(P, T, ye_he(P, x[0], x[1], x[2]));
	else if (!P.adiabatic) ie[p] = (float)x[3];
	lasthit[p] = tick;
}

// The helium update's inputs: per active pair of the tick its summed
// yGdepHI, yGdepHeI, yGdepHeII and heat, and its deposit counter. Runs of
// more than RUN_THREAD hits a warp each (lanes strided, then a fixed
// butterfly), the others a thread each (sorted runs read in order, runs of
// up to short_max put in hit order by visit_run).
__global__ void __launch_bounds__(256) k_sum_he(int t, const int32_t *__restrict__ tick_act,
		const uint32_t *__restrict__ act_ipar, const uint32_t *__restrict__ act_seg, const double *__restrict__ acc,
		const uint32_t *__restrict__ vals, uint32_t short_max, int want_heat, const uint32_t *__restrict__ long_act,
		const int32_t *__restrict__ tick_long, int32_t *__restrict__ hits, double *__restrict__ sum_g0,
		double *__restrict__ sum_g1, double *__restrict__ sum_g2, double *__restrict__ sum_heat) {
	const double2 *acc2 = reinterpret_cast<const double2 *>(acc);
	const int lane = threadIdx.x & 31;
	const int nwarp = (int)((gridDim.x * blockDim.x) >> 5);
	for (int e = tick_long[t] + (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); e < tick_long[t + 1];
			e += nwarp) {
		const int a = (int)long_act[e];
		const uint32_t s0 = act_seg[a], s1 = act_seg[a + 1];
		if (s1 - s0 <= RUN_THREAD) continue;
		double g0 = 0.0, g1 = 0.0, g2 = 0.0, heat = 0.0;
		int nh = 0;
		for (uint32_t k = s0 + lane; k < s1; k += 32) {
			const size_t hk = vals[k];
			const double2 x = acc2[2 * hk];
			if (x.x >= 0.0) {
				const double2 y = acc2[2 * hk + 1];
				g0 += x.x;
				g1 += y.x;
				g2 += y.y;
				if (want_heat) heat += x.y;
				nh++;
			}
		}
#pragma unroll
		for (int o = 16; o > 0; o >>= 1) {
			g0 += __shfl_xor_sync(0xffffffffu, g0, o);
			g1 += __shfl_xor_sync(0xffffffffu, g1, o);
			g2 += __shfl_xor_sync(0xffffffffu, g2, o);
			heat += __shfl_xor_sync(0xffffffffu, heat, o);
			nh += __shfl_xor_sync(0xffffffffu, nh, o);
		}
		if (lane == 0) {
			sum_g0[a] = g0;
			sum_g1[a] = g1;
			sum_g2[a] = g2;
			sum_heat[a] = heat;
			hits[act_ipar[a]] += nh;
		}
	}
	const int hi = tick_act[t + 1];
	for (int a = tick_act[t] + (int)(blockIdx.x * blockDim.x + threadIdx.x); a < hi;
			a += (int)(gridDim.x * blockDim.x)) {
		const uint32_t s0 = act_seg[a], s1 = act_seg[a + 1];
		if (s1 - s0 > RUN_THREAD) continue;
		double g0 = 0.0, g1 = 0.0, g2 = 0.0, heat = 0.0;
		int nh = 0;
		visit_run(vals, s0, s1, short_max, [&](uint32_t h) {
			const size_t hk = h;
			const double2 x = acc2[2 * hk];
			if (x.x >= 0.0) {
				const double2 y = acc2[2 * hk + 1];
				g0 += x.x;
				g1 += y.x;
				g2 += y.y;
				if (want_heat) heat += x.y;
				nh++;
			}
		});
		sum_g0[a] = g0;
		sum_g1[a] = g1;
		sum_g2[a] = g2;
		sum_heat[a] = heat;
		hits[act_ipar[a]] += nh;
	}
}

template <bool REC>
__global__ void __launch_bounds__(128, 4) k_update_he(int t, const int32_t *__restrict__ tick_act,
		const uint32_t *__restrict__ act_ipar, const double *__restrict__ sum_g0, const double *__restrict__ sum_g1,
		const double *__restrict__ sum_g2, const double *__restrict__ sum_heat, double *__restrict__ lambdaH,
		float *__restrict__ ie,
		int64_t *__restrict__ lasthit, const float *__restrict__ rho, const float *__restrict__ yeMET, PhysParams P,
		const PsgBatchDev *__restrict__ B, HeStiffItem *__restrict__ stiff, unsigned *__restrict__ nstiff,
		uint32_t *__restrict__ status) {
	const int64_t tick = B->tick0 + t;
	const double tick_time = B->tick_time;
	const int hi = tick_act[t + 1];
	for (int a = tick_act[t] + (int)(blockIdx.x * blockDim.x + threadIdx.x); a < hi;
			a += (int)(gridDim.x * blockDim.x)) {
	double g0 = sum_g0[a], g1 = sum_g1[a], g2 = sum_g2[a];
	const double heat = sum_heat[a];
	const uint32_t p = act_ipar[a];
	if (P.euler) {      // photons left over by an earlier explicit step (loop.c:745-747)
		g0 += P.gcarry[p];
		g1 += P.gcarryHe1[p];
		g2 += P.gcarryHe2[p];
	}
	HeStep s;
	s.yeMET = (double)yeMET[p];
	s.gHI = g0;
	s.gHeI = g1;
	s.gHeII = g2;
	s.heat = heat;
	s.time = (double)(tick - lasthit[p]) * tick_time;
	s.nH = P.H_PER_MASS * (double)rho[p];
	const double ie0 = (double)ie[p];
	s.T = ieye2T(P, ie0, ye_he(P, lambdaH[p], P.lamHeI[p], P.lamHeII[p]));     // psys_T()
	double x[4] = {lambdaH[p], P.lamHeI[p], P.lamHeII[p], ie0};
	double rec[3] = {0.0, 0.0, 0.0};
	if (P.ygrec) {
		rec[0] = (double)P.ygrec[p];
		rec[1] = (double)P.ygrecHe1[p];
		rec[2] = (double)P.ygrecHe2[p];
	}
	uint32_t st = 0;
	if (P.euler) {
		// step_evolve_euler(): no clamps there; update_pars() clamps
		// (loop.c:759-761) and keeps the unused photons (loop.c:745-747)
		double remain = 0.0, gain[3] = {0.0, 0.0, 0.0};
		int refined = 0;
		st = euler_he(P, s, x, remain, refined, P.ygrec ? gain : nullptr);
		if (P.ygrec)
			for (int k = 0; k < 3; k++) rec[k] += gain[k];
		x[0] = fmax(0.0, fmin(1.0, x[0]));
		x[1] = fmax(0.0, fmin(1.0, x[1]));
		x[2] = fmax(0.0, fmin(1.0 - x[1], x[2]));
		P.gcarry[p] = g0 * remain;
		P.gcarryHe1[p] = g1 * remain;
		P.gcarryHe2[p] = g2 * remain;
	} else {
		double gain[3] = {0.0, 0.0, 0.0}, tt = 0.0, hh = 0.0;
		if (!dopri_he_explicit<REC>(P, s, x, gain, &tt, &hh)) {
			HeStiffItem it;
			it.s = s;
			for (int k = 0; k < 4; k++) it.x[k] = x[k];
			for (int k = 0; k < 3; k++) it.rec[k] = rec[k] + gain[k];
			it.t = tt;
			it.h = hh;
			it.p = p;
			stiff[atomicAdd(nstiff, 1u)] = it;
			continue;
		}
		if (!(x[3] >= 0.0)) st |= PSG_ST_IE_NEG;
		for (int k = 0; k < 4; k++)
			if (!isfinite(x[k])) st |= PSG_ST_NAN;
		clamp_he(x);
		if (P.ygrec)
			for (int k = 0; k < 3; k++) rec[k] = fmax(0.0, rec[k] + gain[k]);
	}
	he_write(P, p, x, rec, s.T, tick, lambdaH, ie, lasthit);
	if (st) atomicOr(status, st);
	}
}

// The stiff helium particles of a tick, one thread each (their number is
// read on the device): the Rosenbrock finish from where the explicit steps
// stopped.
__global__ void __launch_bounds__(64) k_update_he_stiff(const HeStiffItem *__restrict__ stiff,
		const unsigned *__restrict__ nstiff, double *__restrict__ lambdaH, float *__restrict__ ie,
		int64_t *__restrict__ lasthit, PhysParams P, const PsgBatchDev *__restrict__ B, int t,
		uint32_t *__restrict__ status) {
	const int64_t tick = B->tick0 + t;
	const unsigned n = *nstiff;
	uint32_t st = 0;
	for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
		const HeStiffItem &it = stiff[i];
		double x[4] = {it.x[0], it.x[1], it.x[2], it.x[3]};
		double gain[3] = {0.0, 0.0, 0.0}, rec[3];
		if (!rosenbrock_he(P, it.s, x, it.t, it.h, UPD_MAX_STEPS, P.ygrec ? gain : nullptr)) st |= PSG_ST_SOLVER;
		if (!(x[3] >= 0.0)) st |= PSG_ST_IE_NEG;
		for (int k = 0; k < 4; k++)
			if (!isfinite(x[k])) st |= PSG_ST_NAN;
		clamp_he(x);
		for (int k = 0; k < 3; k++) rec[k] = fmax(0.0, it.rec[k] + gain[k]);
		he_write(P, it.p, x, rec, it.s.T, tick, lambdaH, ie, lasthit);
	}
	if (st) atomicOr(status, st);
}

// Update log (training data of the surrogate): the inputs of every active
// particle's step before the update, the outputs after it.
__global__ void k_log_pre(int t, const int32_t *__restrict__ tick_act, const uint32_t *__restrict__ act_ipar,
		const double *__restrict__ act_g, const double *__restrict__ act_heat, const double *__restrict__ lambdaH,
		const float *__restrict__ ie, const int64_t *__restrict__ lasthit, const float *__restrict__ rho,
		const float *__restrict__ yeMET, PhysParams P, const PsgBatchDev *__restrict__ B, float *__restrict__ feat) {
	const int64_t tick = B->tick0 + t;
	const double tick_time = B->tick_time;
	const int lo = tick_act[t], hi = tick_act[t + 1];
	for (int a = lo + (int)(blockIdx.x * blockDim.x + threadIdx.x); a < hi; a += (int)(gridDim.x * blockDim.x)) {
	const uint32_t p = act_ipar[a];
	const double time = rn_dmul((double)(tick - lasthit[p]), tick_time);
	const double lam0 = lambdaH[p], ie0 = (double)ie[p];
	const double T = ieye2T(P, ie0, rn_dadd(rn_dsub(1.0, lam0), P.he_e));
	const RhsCtx cx = make_rhs_ctx(P, (double)yeMET[p], act_g[a], act_heat[a], time,
			rn_dmul(P.H_PER_MASS, (double)rho[p]), T);
	float f[PSG_SURR_NFEAT];
	surr_features(cx, lam0, ie0, f);
	for (int i = 0; i < PSG_SURR_NFEAT; i++) feat[(size_t)(a - lo) * 8 + i] = f[i];
	}
}

__global__ void k_log_post(int t, const int32_t *__restrict__ tick_act, const uint32_t *__restrict__ act_ipar,
		const double *__restrict__ lambdaH, const float *__restrict__ ie, const float *__restrict__ yeMET,
		PhysParams P, const float *__restrict__ feat, float *__restrict__ out, size_t cap,
		unsigned long long *__restrict__ count) {
	const int lo = tick_act[t], hi = tick_act[t + 1];
	for (int a = lo + (int)(blockIdx.x * blockDim.x + threadIdx.x); a < hi; a += (int)(gridDim.x * blockDim.x)) {
	const uint32_t p = act_ipar[a];
	const double lam1 = lambdaH[p];
	const double T1 = ieye2T(P, (double)ie[p], rn_dadd(rn_dsub(1.0, lam1), P.he_e));
	const float *f = feat + (size_t)(a - lo) * 8;
	const float y0 = (float)(surr_logit(lam1) - (double)f[2]);
	const float y1 = (float)(log10(fmax(T1, 1e-300)) - (double)f[1]);
	if (!isfinite(y0) || !isfinite(y1)) continue;
	const unsigned long long row = atomicAdd(count, 1ull);
	if (row >= cap) continue;
	float *o = out + row * 8;
	for (int i = 0; i < PSG_SURR_NFEAT; i++) o[i] = f[i];
	o[5] = y0;
	o[6] = y1;
	o[7] = 0.0f;
	}
}

__global__ void k_step_evolve(psg_step *steps, size_t n, PhysParams P, uint32_t *status) {
	const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
	if (i >= n) return;
	psg_step s = steps[i];
	if (!P.h_only) {
		// step_evolve() with helium (solve.c:170-316)
		HeStep hs;
		hs.yeMET = s.yeMET; hs.gHI = s.yGdepHI; hs.gHeI = s.yGdepHeI; hs.gHeII = s.yGdepHeII;
		hs.heat = s.heat; hs.time = s.time; hs.nH = s.nH; hs.T = s.T;
		double x[4] = {s.lambdaH, s.lambdaHeI, s.lambdaHeII, s.ie};
		double rec[3] = {s.yGrecHII, s.yGrecHeII, s.yGrecHeIII};
		uint32_t st;
		if (P.euler) {
			double remain = 0.0, gain[3] = {0.0, 0.0, 0.0};
			int refined = 0;
			st = euler_he(P, hs, x, remain, refined, P.on_the_spot ? nullptr : gain);
			for (int k = 0; k < 3; k++) rec[k] += gain[k];
			s.step_remain = remain;
			s.refined = refined;
		} else {
			st = solve_step_he(P, hs, x, P.on_the_spot ? nullptr : rec);
			s.step_remain = 0.0;
		}
		s.yGrecHII = rec[0];
		s.yGrecHeII = rec[1];
		s.yGrecHeIII = rec[2];
		s.lambdaH = x[0];
		s.lambdaHeI = x[1];
		s.lambdaHeII = x[2];
		s.ie = x[3];
		steps[i] = s;
		if (st) atomicOr(status, st);
		return;
	}
	if (P.euler) {
		// step_evolve_euler(): no clamping here (update_pars clamps), the
		// unused fraction of the step and whether it was subdivided
		const RhsCtx cx = make_rhs_ctx(P, s.yeMET, s.yGdepHI, s.heat, s.time, s.nH, s.T);
		double x[2] = {s.lambdaH, s.ie};
		double remain = 0.0, grec = 0.0;
		int refined = 0;
		const uint32_t st = P.on_the_spot ? euler_step<false>(P, cx, x, remain, refined)
			: euler_step<true>(P, cx, x, remain, refined, &grec);
		s.lambdaH = x[0];
		s.ie = x[1];
		s.yGrecHII += grec;
		s.step_remain = remain;
		s.refined = refined;
		steps[i] = s;
		if (st) atomicOr(status, st);
		return;
	}
	double lam = s.lambdaH, e = s.ie, grec = 0.0;
	const uint32_t st = solve_step(P, lam, e, s.yeMET, s.yGdepHI, s.heat, s.time, s.nH, s.T, &grec);
	s.lambdaH = lam;
	s.ie = e;
	if (!P.on_the_spot) s.yGrecHII = fmax(0.0, s.yGrecHII + grec);      // x[3] of solve.c:183,211,218
	s.step_remain = 0.0;
	steps[i] = s;
	if (st) atomicOr(status, st);
}

}  // namespace

static int check_status(psg_context *ctx) {
	uint32_t st = 0;
	PSG_CUDA(cudaMemcpyAsync(&st, ctx->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
	PSG_CUDA(cudaStreamSynchronize(ctx->stream));
	if (st) {
		PSG_CUDA(cudaMemsetAsync(ctx->d_status, 0, sizeof(uint32_t), ctx->stream));
		return psg_fail(ctx, PSG_E_DEVICE, "device status 0x%x:%s%s%s", st,
				(st & PSG_ST_NAN) ? " non-finite state" : "",
				(st & PSG_ST_SOLVER) ? " integrator step limit" : "",
				(st & PSG_ST_IE_NEG) ? " negative internal energy" : "");
	}
	return PSG_OK;
}

// ---- one batch of ticks on the host side -------------------------------------
//
// A batch is: the traversal of all its rays (psg_trace_fill), then one host
// synchronisation that reads the hit total; everything after it -- the
// per-ray sort, the by-particle order, the ray and particle classes and the
// K ticks of deposit and update -- is issued by enqueue_batch() with sizes
// fixed by the batch's shape and buffer capacities, counts read on the
// device, and no allocation. That part is captured once as a CUDA graph and
// replayed for every later batch of the same shape (first tick, tick length
// and rays are read from ctx->d_batch). A last synchronisation reads the
// counters and the status word: two per batch.

__global__ void k_set_batch(PsgBatchDev *b, int64_t tick0, double tick_time, const psg_ray *rays,
		const psg_ray *src) {
	b->tick0 = tick0;
	b->tick_time = tick_time;
	b->rays = rays;
	b->src = src;
	b->k = 0;
}

namespace {

// Buffers and sizes of one batch, all fixed before anything is issued.
struct BatchPlan {
	size_t R = 0, K = 0, nray = 0;
	size_t nhit = 0;            // the batch's hits (used only by the long-list sort, which is never captured)
	size_t cap = 0;             // hits the per-hit buffers hold (>= the batch's hits)
	size_t pcap = 0;            // particles one tick can update (min(n, cap))
	unsigned long long maxcount = 0;
	size_t KN = 0;              // slot keys: ticks x particles
	int long_cap = 0;           // longest run of one particle's hits the slot order sorts in shared memory
	int nacc = 1, want_heat = 0;
	bool gen = false, helium = false, iso = false, euler = false, surr = false, aff = false, feat_on = false;

	// grids
	unsigned dep_grid = 0, red_grid = 0, queue_grid = 0, he_grid = 0, euler_grid = 0, log_grid = 0;
	int queue_minb = 1;         // the integrator's register limit: resident blocks per SM
	size_t src_R = 0;           // > 0: a recombination tick whose first src_R rays come traced and sorted (S_SRCHIT)
};

struct GraphEntry {
	std::vector<unsigned long long> key;
	cudaGraphExec_t exec = nullptr;
	long launches = 0;
};
struct GraphCache {
	std::vector<GraphEntry> e;
};

template <typename KF>
unsigned occ_grid(const psg_context *ctx, KF kern, int threads, size_t smem = 0) {
	int per_sm = 1;
	if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem) != cudaSuccess) {
		cudaGetLastError();
		per_sm = 1;
	}
	return (unsigned)(std::max(per_sm, 1) * ctx->sms);
}

// Layout of the per-batch scratch slots.
struct ActView {
	uint32_t *act_ipar, *act_seg;
	int32_t *tick_act;
};
ActView act_view(psg_context *ctx, const BatchPlan &pl) {
	ActView v;
	char *actm = (char *)ctx->scratch[S_ACT].p;
	v.act_ipar = (uint32_t *)actm;
	v.act_seg = v.act_ipar + (pl.cap + 1);
	v.tick_act = (int32_t *)(((uintptr_t)(v.act_seg + pl.cap + 1) + 15) & ~(uintptr_t)15);
	return v;
}
size_t act_bytes(const BatchPlan &pl) { return sizeof(uint32_t) * 2 * (pl.cap + 1) + sizeof(int32_t) * (pl.K + 2) + 64; }
// S_SLOTCNT: the per-key counters (K * N, u32), then the keys' scan (K * N + 1, u64)
size_t slotcnt_bytes(const BatchPlan &pl) { return 16 * ((4 * pl.KN + 15) / 16) + 8 * (pl.KN + 1) + 64; }
unsigned long long *slot_base(psg_context *ctx, const BatchPlan &pl) {
	return (unsigned long long *)((char *)ctx->scratch[S_SLOTCNT].p + 16 * ((4 * pl.KN + 15) / 16));
}
// S_ALONG: the long pairs (at most cap/33 + 1; cap + 1 reserved), the
// middle and very long ones, each tick's first long pair (K + 1), then,
// zeroed per batch, the per-tick counts and their scan (K + 1, u64), the
// per-tick cursors and the two list counts.
struct LongLists {
	uint32_t *long_act, *mid_list, *vl_list;
	int32_t *tick_long;
	unsigned long long *tick_off;
	unsigned *cursor, *mid_count, *vl_count;
	void *zero;
	size_t zero_bytes;
};
LongLists long_lists_at(char *m, size_t cap, size_t K, size_t *bytes) {
	auto up = [](size_t x) { return (x + 255) & ~(size_t)255; };
	LongLists l;
	size_t o = 0;
	l.long_act = (uint32_t *)(m + o); o = up(o + sizeof(uint32_t) * (cap + 1));
	l.mid_list = (uint32_t *)(m + o); o = up(o + sizeof(uint32_t) * (cap / SLOT_WARP_MAX + 2));
	l.vl_list = (uint32_t *)(m + o); o = up(o + sizeof(uint32_t) * (cap / SLOT_MID_MAX + 2));
	l.tick_long = (int32_t *)(m + o); o = up(o + sizeof(int32_t) * (K + 1));
	const size_t z0 = o;
	l.tick_off = (unsigned long long *)(m + o); o += sizeof(unsigned long long) * (K + 1);
	l.cursor = (unsigned *)(m + o); o += sizeof(unsigned) * (K + 1);
	l.vl_count = (unsigned *)(m + o); o += sizeof(unsigned);
	l.mid_count = (unsigned *)(m + o); o += sizeof(unsigned);
	l.zero = m + z0;
	l.zero_bytes = o - z0;
	o = up(o);
	if (bytes) *bytes = o;
	return l;
}
LongLists long_lists(psg_context *ctx, const BatchPlan &pl) {
	return long_lists_at((char *)ctx->scratch[S_ALONG].p, pl.cap, pl.K, nullptr);
}
size_t long_lists_bytes(const BatchPlan &pl) {
	size_t b = 0;
	long_lists_at(nullptr, pl.cap, pl.K, &b);
	return b;
}
struct UpdView {
	double *act_g, *act_heat;
	unsigned *cursors, *nstiff, *nrej, *dep_ctr, *cursors2;
	TickRays *tick_rays;
	StiffItem *stiff;
	uint32_t *rej;
	uint8_t *act_slow;        // not isothermal: per active pair, the integrator's first pass
};
UpdView upd_view(psg_context *ctx, const BatchPlan &pl) {
	UpdView v;
	char *um = (char *)ctx->scratch[S_UPD].p;
	v.act_g = (double *)um;
	v.act_heat = v.act_g + pl.cap;
	// (with helium two more per-pair sums follow act_heat: yGdepHeI, yGdepHeII)
	v.cursors = (unsigned *)(v.act_heat + pl.cap * (pl.helium ? 3 : 1));
	v.nstiff = v.cursors + (pl.K + 1);
	v.nrej = v.nstiff + (pl.K + 1);
	v.dep_ctr = v.nrej + (pl.K + 1);
	v.cursors2 = v.dep_ctr + (pl.K + 1);       // the integrator's second pass (update_order)
	v.tick_rays = (TickRays *)(((uintptr_t)(v.cursors2 + pl.K + 1) + 31) & ~(uintptr_t)31);
	v.stiff = (StiffItem *)(((uintptr_t)(v.tick_rays + pl.K) + 15) & ~(uintptr_t)15);
	v.rej = (uint32_t *)(v.stiff + (pl.iso ? 0 : pl.pcap));
	v.act_slow = (uint8_t *)(v.rej + (pl.surr ? pl.pcap : 0));
	return v;
}
size_t upd_bytes(const BatchPlan &pl) {
	return sizeof(double) * (pl.helium ? 4 : 2) * pl.cap + sizeof(unsigned) * 5 * (pl.K + 1) + sizeof(TickRays) * pl.K +
			(pl.iso ? 0 : sizeof(StiffItem) * pl.pcap + pl.cap) + (pl.surr ? sizeof(uint32_t) * pl.pcap : 0) + 512;
}

// Sizes, capacities and every buffer of the batch (allocates; before any
// capture). tf: the traversal's totals.
int plan_batch(psg_context *ctx, size_t R, size_t K, const PsgTraceFill &tf, BatchPlan &pl) {
	pl.R = R;
	pl.K = K;
	pl.nray = R * K;
	pl.maxcount = tf.maxcount;
	pl.nhit = tf.nhit;
	// grow-only capacity with an eighth of headroom, so batches of similar
	// hit counts share one captured graph
	if (tf.nhit > ctx->batch_cap) {
		size_t c = tf.nhit + tf.nhit / 8;
		c = (c + 65535) & ~(size_t)65535;
		ctx->batch_cap = c;
	}
	pl.cap = std::max<size_t>(ctx->batch_cap, 1);
	pl.pcap = std::max<size_t>(std::min(ctx->n, pl.cap), 1);
	pl.KN = K * ctx->n;
	if (pl.KN >= (1ull << 31))
		return psg_fail(ctx, PSG_E_OVERFLOW, "psg_run_ticks: %zu ticks x %zu particles: fewer ticks per call", K,
				ctx->n);
	{
		int P = 1;
		while (P < (int)std::min<size_t>(R, SLOT_LONG_MAX)) P <<= 1;
		pl.long_cap = P;
	}
	pl.want_heat = !ctx->flags.isothermal;
	pl.gen = !ctx->flags.h_only || ctx->flags.secondary_ionization;
	pl.helium = !ctx->flags.h_only;
	pl.nacc = pl.helium ? 4 : (pl.want_heat ? 2 : 1);
	pl.iso = ctx->flags.isothermal != 0;
	pl.euler = ctx->flags.euler != 0;
	// (the network does not model the recombination photons: on the spot only)
	pl.surr = !pl.iso && !pl.euler && ctx->surr_on && !ctx->flags.adiabatic && ctx->flags.on_the_spot &&
			ctx->flags.h_only;
	pl.feat_on = ctx->log_buf && !pl.iso && !pl.helium;
	// capped hits settled by the affine-map scan when the last batch had many
	pl.aff = ctx->sat_frac > 1e-3;
	const size_t cap = pl.cap, nray = pl.nray;

	int rc = psg_trace_sort_prepare(ctx, nray, cap, pl.maxcount);
	if (rc) return rc;
	// slots and the active lists
	if (!psg_scratch(ctx, S_VALS, sizeof(uint32_t) * 2 * cap) ||
			!psg_scratch(ctx, S_ACC, sizeof(double) * cap * pl.nacc) || !psg_scratch(ctx, S_ACT, act_bytes(pl)) ||
			!psg_scratch(ctx, S_SLOTCNT, slotcnt_bytes(pl)))
		return PSG_E_NOMEM;
	if (std::max(pl.long_cap, 2048) * sizeof(uint32_t) > 48 * 1024)
		PSG_CUDA(cudaFuncSetAttribute(k_slot_canon_long, cudaFuncAttributeMaxDynamicSharedMemorySize,
				(int)(std::max(pl.long_cap, 2048) * sizeof(uint32_t))));
	// ray classes (S_COUNT: class flags and scan; S_RAYLIST: the three lists,
	// a room of nray each, inside the sort's class lists)
	if (!psg_scratch(ctx, S_COUNT, sizeof(unsigned long long) * 2 * (nray + 1))) return PSG_E_NOMEM;
	if (ctx->scratch[S_RAYLIST].bytes < sizeof(uint32_t) * 3 * (nray + 1)) return PSG_E_NOMEM;
	// updates
	if (!psg_scratch(ctx, S_UPD, upd_bytes(pl)) ||
			!psg_scratch(ctx, S_ALONG, long_lists_bytes(pl)))
		return PSG_E_NOMEM;
	if (pl.helium) {
		if (!psg_scratch(ctx, S_REC, sizeof(HeStiffItem) * pl.pcap)) return PSG_E_NOMEM;
	} else if (pl.euler) {
		if (!psg_scratch(ctx, S_REC, sizeof(UpdRec) * pl.pcap)) return PSG_E_NOMEM;
	}
	if (pl.feat_on && !psg_scratch(ctx, S_LOG, sizeof(float) * 8 * pl.pcap)) return PSG_E_NOMEM;
	// the scans' tile sums (one buffer, scans one after another in stream order)
	if (!psg_scratch(ctx, S_SCAN, sizeof(unsigned long long) * (scan_tiles(std::max(std::max(pl.KN, cap + 1),
			nray + 1)) + 1)))
		return PSG_E_NOMEM;
	// grids of the persistent kernels
	pl.dep_grid = pl.gen ? occ_grid(ctx, k_deposit<true, false>, DEP_THREADS)
			: (pl.aff ? occ_grid(ctx, k_deposit<false, true>, DEP_THREADS) : occ_grid(ctx, k_deposit<false, false>,
					DEP_THREADS));
	pl.red_grid = occ_grid(ctx, k_reduce<false, false>, 256);
	pl.queue_minb = ctx->tune.update_minblocks >= 4 ? 4 : (ctx->tune.update_minblocks == 3 ? 3 : 1);
	pl.queue_grid = pl.queue_minb == 4 ? occ_grid(ctx, k_update_queue<false, 4>, 32 * UPD_WARPS)
			: pl.queue_minb == 3 ? occ_grid(ctx, k_update_queue<false, 3>, 32 * UPD_WARPS)
			: occ_grid(ctx, k_update_queue<false, 1>, 32 * UPD_WARPS);
	pl.he_grid = occ_grid(ctx, k_update_he<false>, 128);
	pl.euler_grid = occ_grid(ctx, k_update_euler, 128);
	pl.log_grid = (unsigned)(ctx->sms * 8);
	if (pl.surr) {
		rc = psg_surrogate_prepare(ctx);
		if (rc) return rc;
	}
	return PSG_OK;
}

// Everything of the batch after the traversal. No host reads, no
// allocation: the launch shapes depend on the plan alone; per-call values
// come from B.
int enqueue_batch(psg_context *ctx, const BatchPlan &pl, const PsgBatchDev *B) {
	cudaStream_t st = ctx->stream;
	const size_t R = pl.R, K = pl.K, nray = pl.nray, cap = pl.cap;
	const PhysParams P = psg_phys_params(ctx);
	const int sms = ctx->sms;
	int rc = pl.src_R ? psg_trace_rec_sort_enqueue(ctx, pl.src_R, nray, pl.maxcount, B)
			: psg_trace_sort_enqueue(ctx, nray, pl.nhit, pl.maxcount, 1, 0);
	if (rc) return rc;
	int64_t *off64 = (int64_t *)ctx->scratch[S_OFFSETS].p;
	uint32_t *hit_ipar = (uint32_t *)ctx->scratch[S_HIT_IPAR].p;
	double *hit_kern = (double *)ctx->scratch[S_HIT_KERN].p;

	// by-particle order of all hits: per (tick, particle) key its run of
	// slots, counted, placed, then put in hit order
	psg_mark_begin(ctx, PSG_K_SLOTS);
	uint32_t *vals = (uint32_t *)ctx->scratch[S_VALS].p;
	double *acc = (double *)ctx->scratch[S_ACC].p;
	ActView av = act_view(ctx, pl);
	uint32_t *kcnt = (uint32_t *)ctx->scratch[S_SLOTCNT].p;
	unsigned long long *kbase = slot_base(ctx, pl);
	unsigned long long *tiles = (unsigned long long *)ctx->scratch[S_SCAN].p;
	const uint32_t N = (uint32_t)ctx->n;
	const unsigned cgrid = (unsigned)std::min<size_t>(blocks(cap, 256), (size_t)sms * 16);
	PSG_CUDA(cudaMemsetAsync(kcnt, 0, sizeof(uint32_t) * pl.KN, st));
	k_slot_count<<<blocks(nray * 32, 256), 256, 0, st>>>(nray, (int)R, N, off64, hit_ipar, kcnt);
	PSG_CHECK_LAUNCH();
	PSG_CUDA(scan_enqueue(st, kcnt, pl.KN, kbase, tiles, SlotPair()));
	unsigned long long *d_nact = ctx->d_counters + 6;
	k_act_build<<<(unsigned)std::min<size_t>(blocks(pl.KN, 256), (size_t)sms * 16), 256, 0, st>>>(pl.KN, N, (int)K,
			kbase, av.act_ipar, av.act_seg, av.tick_act, d_nact, kcnt);
	PSG_CHECK_LAUNCH();
	k_slot_place<<<blocks(nray * 32, 256), 256, 0, st>>>(nray, (int)R, N, off64, hit_ipar, kcnt, vals);
	PSG_CHECK_LAUNCH();
	ctx->launches += 8;
	unsigned long long *d_nsat = ctx->d_counters + 1;      // (zeroed by the caller, per call)
	psg_mark_end(ctx);

	// long / middle / short ray lists of the batch (ray order, so each
	// tick's rays are a run of each), and each tick's ranges in them
	unsigned long long *cls = (unsigned long long *)ctx->scratch[S_COUNT].p;
	unsigned long long *cls_scan = cls + (nray + 1);
	uint32_t *ray_lists = (uint32_t *)ctx->scratch[S_RAYLIST].p;
	uint32_t *long_rays = ray_lists, *mid_rays = ray_lists + nray, *short_rays = ray_lists + 2 * nray;
	UpdView uv = upd_view(ctx, pl);
	k_ray_class<<<blocks(nray, 256), 256, 0, st>>>(nray, off64, ctx->tune.deposit_long, ctx->tune.deposit_mid, cls);
	PSG_CHECK_LAUNCH();
	PSG_CUDA(scan_enqueue(st, cls, nray, cls_scan, tiles, Widen()));
	k_ray_lists<<<blocks(nray, 256), 256, 0, st>>>(nray, cls, cls_scan, long_rays, mid_rays, short_rays);
	PSG_CHECK_LAUNCH();
	k_tick_rays<<<blocks(K, 128), 128, 0, st>>>((int)K, R, nray, cls, cls_scan, uv.tick_rays);
	PSG_CHECK_LAUNCH();
	ctx->launches += 3;

	// the long-segment lists and (not isothermal) the integrator's work
	// cursors, stiff lists and the deposit's unit counters
	PSG_CUDA(cudaMemsetAsync(uv.cursors, 0, sizeof(unsigned) * 5 * (K + 1), st));
	if (pl.surr) PSG_CUDA(cudaMemsetAsync(ctx->d_counters + 8, 0, sizeof(unsigned long long), st));
	UpdRec *urec = (!pl.helium && pl.euler) ? (UpdRec *)ctx->scratch[S_REC].p : nullptr;
	HeStiffItem *hstiff = pl.helium ? (HeStiffItem *)ctx->scratch[S_REC].p : nullptr;
	float *feat = pl.feat_on ? (float *)ctx->scratch[S_LOG].p : nullptr;
	LongLists ll = long_lists(ctx, pl);
	PSG_CUDA(cudaMemsetAsync(ll.zero, 0, ll.zero_bytes, st));
	k_long_count<<<cgrid, 256, 0, st>>>(av.tick_act, (int)K, av.act_seg, (uint32_t)ctx->tune.run_short, ll.tick_off);
	PSG_CHECK_LAUNCH();
	k_scan_sums<unsigned long long><<<1, 1024, 0, st>>>(ll.tick_off, K);
	PSG_CHECK_LAUNCH();
	k_long_place<<<cgrid, 256, 0, st>>>(av.tick_act, (int)K, av.act_seg, (uint32_t)ctx->tune.run_short, ll.tick_off,
			ll.cursor, ll.long_act,
			ll.tick_long, ll.mid_list, ll.mid_count, ll.vl_list, ll.vl_count);
	PSG_CHECK_LAUNCH();
	int32_t *tick_long = ll.tick_long;
	uint32_t *long_act = ll.long_act;
	// the slot order of the long runs (the short ones are in order already)
	psg_mark_begin(ctx, PSG_K_SLOTS);
	k_slot_canon_warp<<<(unsigned)(4 * sms), 32 * SLOT_WARPS, 0, st>>>(tick_long, (int)K, long_act, av.act_seg,
			vals);
	PSG_CHECK_LAUNCH();
	// (a particle's run of one tick holds at most the tick's R hits: the
	// block tiers are launched only where R reaches them)
	if (R > SLOT_WARP_MAX) {
		k_slot_canon_mid<<<(unsigned)(4 * sms), 256, 0, st>>>(ll.mid_list, ll.mid_count, av.act_seg, vals);
		PSG_CHECK_LAUNCH();
	}
	if (R > SLOT_MID_MAX) {
		k_slot_canon_long<<<(unsigned)sms, 1024, sizeof(uint32_t) * std::max(pl.long_cap, 2048), st>>>(ll.vl_list,
				ll.vl_count, av.act_seg, vals, pl.long_cap, cap);
		PSG_CHECK_LAUNCH();
	}
	psg_mark_end(ctx);
	ctx->launches += 6;

	// the tick loop
	double *d_lost = (double *)(ctx->d_counters + 2);
	for (size_t t = 0; t < K; t++) {
		psg_mark_begin(ctx, PSG_K_DEPOSIT);
		if (pl.gen)
			k_deposit<true, false><<<pl.dep_grid, DEP_THREADS, 0, st>>>((int)t, uv.tick_rays, uv.dep_ctr, B,
					long_rays, mid_rays, short_rays, off64, hit_ipar, hit_kern, ctx->d_lambdaH, ctx->d_mass, P,
					pl.want_heat, acc, pl.nacc, d_nsat, d_lost);
		else if (pl.aff)
			k_deposit<false, true><<<pl.dep_grid, DEP_THREADS, 0, st>>>((int)t, uv.tick_rays, uv.dep_ctr, B,
					long_rays, mid_rays, short_rays, off64, hit_ipar, hit_kern, ctx->d_lambdaH, ctx->d_mass, P,
					pl.want_heat, acc, pl.nacc, d_nsat, d_lost);
		else
			k_deposit<false, false><<<pl.dep_grid, DEP_THREADS, 0, st>>>((int)t, uv.tick_rays, uv.dep_ctr, B,
					long_rays, mid_rays, short_rays, off64, hit_ipar, hit_kern, ctx->d_lambdaH, ctx->d_mass, P,
					pl.want_heat, acc, pl.nacc, d_nsat, d_lost);
		PSG_CHECK_LAUNCH();
		ctx->launches++;
		psg_mark_end(ctx);
		psg_mark_begin(ctx, PSG_K_UPDATE);
		if (pl.helium) {
			double *g1 = uv.act_heat + pl.cap, *g2 = g1 + pl.cap;
			k_sum_he<<<pl.red_grid, 256, 0, st>>>((int)t, av.tick_act, av.act_ipar, av.act_seg, acc, vals,
					(uint32_t)ctx->tune.run_short, pl.want_heat, long_act, tick_long, ctx->d_hits, uv.act_g, g1, g2, uv.act_heat);
			PSG_CHECK_LAUNCH();
			ctx->launches++;
			if (P.ygrec)
				k_update_he<true><<<pl.he_grid, 128, 0, st>>>((int)t, av.tick_act, av.act_ipar, uv.act_g, g1, g2,
						uv.act_heat, ctx->d_lambdaH, ctx->d_ie, ctx->d_lasthit, ctx->d_rho,
						ctx->d_yeMET, P, B, hstiff, uv.nstiff + t, ctx->d_status);
			else
				k_update_he<false><<<pl.he_grid, 128, 0, st>>>((int)t, av.tick_act, av.act_ipar, uv.act_g, g1, g2,
						uv.act_heat, ctx->d_lambdaH, ctx->d_ie, ctx->d_lasthit, ctx->d_rho,
						ctx->d_yeMET, P, B, hstiff, uv.nstiff + t, ctx->d_status);
			PSG_CHECK_LAUNCH();
			k_update_he_stiff<<<sms, 64, 0, st>>>(hstiff, uv.nstiff + t, ctx->d_lambdaH, ctx->d_ie, ctx->d_lasthit,
					P, B, (int)t, ctx->d_status);
			PSG_CHECK_LAUNCH();
			ctx->launches += 2;
		} else {
			const double *gcarry = pl.euler ? ctx->d_gcarry : nullptr;
			// not isothermal, every pair's sums first (a thread per short run,
			// a warp per long one): the integrator then reads two doubles per
			// particle instead of gathering its deposits in its latency-bound
			// loop
			double *keep_g = pl.iso ? nullptr : uv.act_g;
			double *keep_heat = pl.iso ? nullptr : uv.act_heat;
			// the integrator's two passes (update_order; not over the surrogate's rejects)
			const bool two_pass = !pl.iso && !pl.euler && ctx->tune.update_order && !pl.surr;
			uint8_t *slow_flags = two_pass ? uv.act_slow : nullptr;
#define PSG_REDUCE(ISO_, REC_)                                                                                 \
	k_reduce<ISO_, REC_><<<pl.red_grid, 256, 0, st>>>((int)t, av.tick_act, av.act_ipar, av.act_seg, acc, vals,\
			(uint32_t)ctx->tune.run_short, pl.want_heat, long_act, tick_long, ctx->d_hits, keep_g, keep_heat, ctx->d_lambdaH, ctx->d_ie,       \
			ctx->d_lasthit, ctx->d_rho, ctx->d_yeMET, ctx->d_hstep, urec, gcarry, slow_flags, P, B, ctx->d_status)
			if (pl.iso && !pl.euler) {
				if (P.ygrec) PSG_REDUCE(true, true);
				else PSG_REDUCE(true, false);
			} else {
				if (P.ygrec) PSG_REDUCE(false, true);
				else PSG_REDUCE(false, false);
			}
#undef PSG_REDUCE
			PSG_CHECK_LAUNCH();
			ctx->launches++;
			if (pl.euler) {
				k_update_euler<<<pl.euler_grid, 128, 0, st>>>((int)t, av.tick_act, urec, ctx->d_lambdaH, ctx->d_ie,
						ctx->d_lasthit, ctx->d_gcarry, P, B, ctx->d_status);
				PSG_CHECK_LAUNCH();
				ctx->launches++;
			} else if (!pl.iso) {
				UpdSrc us;
				us.act_ipar = av.act_ipar;
				us.act_g = uv.act_g;
				us.act_heat = uv.act_heat;
				us.rho = ctx->d_rho;
				us.yeMET = ctx->d_yeMET;
				us.slow = slow_flags;
				if (feat) {
					k_log_pre<<<pl.log_grid, 256, 0, st>>>((int)t, av.tick_act, av.act_ipar, uv.act_g, uv.act_heat,
							ctx->d_lambdaH, ctx->d_ie, ctx->d_lasthit, ctx->d_rho, ctx->d_yeMET, P, B, feat);
					PSG_CHECK_LAUNCH();
				}
				if (pl.surr) {
					// the network first; the integrator takes its rejects
					rc = psg_surrogate_tick(ctx, (int)t, av.tick_act, av.act_ipar, uv.act_g, uv.act_heat, P, B, uv.rej,
							uv.nrej + t);
					if (rc) return rc;
					ctx->launches++;
				}
				unsigned *cur2 = two_pass ? uv.cursors2 + t : nullptr;
				if (P.ygrec) {
					k_update_queue<true, 1><<<pl.queue_grid, 32 * UPD_WARPS, 0, st>>>((int)t, av.tick_act, us,
							ctx->d_lambdaH, ctx->d_ie, ctx->d_lasthit, ctx->d_hstep, P, B, uv.cursors + t, cur2,
							uv.stiff, uv.nstiff + t, nullptr, nullptr, ctx->d_status);
					PSG_CHECK_LAUNCH();
					k_update_stiff<true><<<sms, 64, 0, st>>>(uv.stiff, uv.nstiff + t, ctx->d_lambdaH, ctx->d_ie,
							ctx->d_lasthit, P, B, (int)t, ctx->d_status);
				} else {
#define PSG_QUEUE(MINB_)                                                                                       \
	k_update_queue<false, MINB_><<<pl.queue_grid, 32 * UPD_WARPS, 0, st>>>((int)t, av.tick_act, us,          \
			ctx->d_lambdaH, ctx->d_ie, ctx->d_lasthit, ctx->d_hstep, P, B, uv.cursors + t, cur2, uv.stiff,     \
			uv.nstiff + t, pl.surr ? uv.rej : nullptr, pl.surr ? uv.nrej + t : nullptr, ctx->d_status)
					if (pl.queue_minb == 4) PSG_QUEUE(4);
					else if (pl.queue_minb == 3) PSG_QUEUE(3);
					else PSG_QUEUE(1);
#undef PSG_QUEUE
					PSG_CHECK_LAUNCH();
					k_update_stiff<false><<<sms, 64, 0, st>>>(uv.stiff, uv.nstiff + t, ctx->d_lambdaH, ctx->d_ie,
							ctx->d_lasthit, P, B, (int)t, ctx->d_status);
				}
				PSG_CHECK_LAUNCH();
				ctx->launches += 2;
				if (feat) {
					k_log_post<<<pl.log_grid, 256, 0, st>>>((int)t, av.tick_act, av.act_ipar, ctx->d_lambdaH,
							ctx->d_ie, ctx->d_yeMET, P, feat, ctx->log_buf, ctx->log_cap, ctx->log_count);
					PSG_CHECK_LAUNCH();
				}
			}
		}
		psg_mark_end(ctx);
	}
	return PSG_OK;
}

// What a captured batch depends on: the plan, every buffer address, the
// physics (PhysParams by value), the launch shapes and the surrogate and log
// settings.
std::vector<unsigned long long> batch_key(const psg_context *ctx, const BatchPlan &pl, const PsgBatchDev *B) {
	std::vector<unsigned long long> k;
	k.push_back(pl.R); k.push_back(pl.K); k.push_back(pl.cap); k.push_back(pl.pcap);
	k.push_back(pl.maxcount > PSG_SORT_MAX); k.push_back(pl.KN); k.push_back((unsigned long long)pl.long_cap);
	k.push_back((unsigned long long)pl.nacc | (pl.want_heat << 4) | (pl.gen << 5) | (pl.helium << 6) | (pl.iso << 7) |
			(pl.euler << 8) | (pl.surr << 9) | (pl.aff << 10) | (pl.feat_on << 11));
	k.push_back((unsigned long long)(uintptr_t)ctx->stream);
	k.push_back((unsigned long long)(uintptr_t)B);
	for (int sl = 0; sl < S_NSLOTS; sl++) {
		k.push_back((unsigned long long)(uintptr_t)ctx->scratch[sl].p);
		k.push_back(ctx->scratch[sl].bytes);
	}
	k.push_back(ctx->slab_cap);
	const PhysParams P = psg_phys_params(ctx);
	const unsigned char *pb = (const unsigned char *)&P;
	for (size_t i = 0; i < sizeof(P); i += 8) {
		unsigned long long v = 0;
		memcpy(&v, pb + i, std::min<size_t>(8, sizeof(P) - i));
		k.push_back(v);
	}
	k.push_back((unsigned long long)(uintptr_t)ctx->d_surr);
	unsigned tolbits = 0;
	memcpy(&tolbits, &ctx->surr_tol, 4);
	k.push_back(tolbits);
	k.push_back((unsigned long long)(uintptr_t)ctx->log_buf);
	k.push_back(ctx->log_cap);
	k.push_back((unsigned long long)(uintptr_t)ctx->log_count);
	const void *dev[] = {ctx->d_psml, ctx->d_order, ctx->d_mass, ctx->d_rho, ctx->d_yeMET, ctx->d_ie, ctx->d_lambdaH,
		ctx->d_hits, ctx->d_lasthit, ctx->d_hstep, ctx->d_gcarry, ctx->d_status, ctx->d_counters};
	for (const void *q : dev) k.push_back((unsigned long long)(uintptr_t)q);
	k.push_back(ctx->n);
	k.push_back(ctx->hit_cap);
	k.push_back((unsigned long long)ctx->tune.deposit_long << 32 | (unsigned)ctx->tune.deposit_mid);
	k.push_back((unsigned long long)pl.queue_minb);
	k.push_back((unsigned long long)ctx->tune.run_short);
	k.push_back((unsigned long long)ctx->tune.update_order);
	k.push_back((unsigned long long)psg_sort_classes(pl.maxcount));
	k.push_back(pl.src_R);
	k.push_back(ctx->src_nray);
	k.push_back(ctx->src_nhit);
	return k;
}

int enqueue_any(psg_context *ctx, const BatchPlan &pl, const PsgBatchDev *B) {
	return enqueue_batch(ctx, pl, B);
}

// Replays the graph of `key`, capturing what `enqueue` issues first if no
// graph of this key exists. A failed capture is discarded before anything
// of it runs. times: how many launches of the graph.
template <typename F>
int launch_graph(psg_context *ctx, std::vector<unsigned long long> key, F enqueue, size_t times = 1) {
	GraphCache *gc = (GraphCache *)ctx->graphs;
	if (!gc) {
		gc = new GraphCache();
		ctx->graphs = gc;
	}
	GraphEntry *hit = nullptr;
	for (auto &e : gc->e)
		if (e.key == key) hit = &e;
	cudaStream_t st = ctx->stream;
	if (!hit) {
		PSG_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
		const long l0 = ctx->launches;
		const int rc = enqueue();
		cudaGraph_t g = nullptr;
		const cudaError_t ec = cudaStreamEndCapture(st, &g);
		if (rc || ec != cudaSuccess) {
			if (g) cudaGraphDestroy(g);
			cudaGetLastError();
			ctx->launches = l0;
			return rc ? rc : psg_cuda_fail(ctx, ec, "cudaStreamEndCapture", __FILE__, __LINE__);
		}
		GraphEntry e;
		e.key = std::move(key);
		e.launches = ctx->launches - l0;
		ctx->launches = l0;
		const cudaError_t ei = cudaGraphInstantiate(&e.exec, g, 0);
		cudaGraphDestroy(g);
		if (ei != cudaSuccess) return psg_cuda_fail(ctx, ei, "cudaGraphInstantiate", __FILE__, __LINE__);
		if (gc->e.size() >= 6) {
			cudaGraphExecDestroy(gc->e.front().exec);
			gc->e.erase(gc->e.begin());
		}
		gc->e.push_back(std::move(e));
		hit = &gc->e.back();
	}
	for (size_t i = 0; i < times; i++) {
		PSG_CUDA(cudaGraphLaunch(hit->exec, st));
		ctx->launches += hit->launches;
	}
	return PSG_OK;
}

// ---- recombination ticks without host reads -----------------------------------
// The ticks of a call not on the spot, each: the tick's source rays into
// the ray buffer, the recombination rays emitted behind them (their count
// stays on the device), the traversal of all of them up to that count, the
// batch of one tick, the next tick's emitter marks, the counters and the
// tick number advanced on the device. Captured once, launched once per
// tick; the host waits once per call.
__global__ void k_rec_src(const PsgBatchDev *__restrict__ B, size_t R, psg_ray *__restrict__ buf) {
	const psg_ray *src = B->src + (size_t)B->k * R;
	for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < R; i += (size_t)gridDim.x * blockDim.x)
		buf[i] = src[i];
}
__global__ void k_rec_tick_end(const int64_t *__restrict__ off, size_t nray, unsigned long long *__restrict__ hitsum,
		PsgBatchDev *__restrict__ B) {
	*hitsum += (unsigned long long)off[nray];
	B->tick0 += 1;
	B->k += 1;
}

}  // namespace

void psg_graphs_free(psg_context *ctx) {
	GraphCache *gc = (GraphCache *)ctx->graphs;
	if (!gc) return;
	for (auto &e : gc->e)
		if (e.exec) cudaGraphExecDestroy(e.exec);
	delete gc;
	ctx->graphs = nullptr;
}

// One batch of K ticks of R rays each, rays already traced together: the
// path on the spot (and the per-tick step of the recombination loop).
int psg_run_ticks_core(psg_context *ctx, const psg_ray *d_rays, size_t R, size_t K,
		int64_t first_tick, double tick_time, psg_tick_stats *stats) {
	if (!ctx) return PSG_E_INVAL;
	if (!ctx->have_physics || !ctx->have_tree)
		return psg_fail(ctx, PSG_E_INVAL, "psg_run_ticks: set physics, load particles and build the tree first");
	if (R == 0 || K == 0 || !d_rays) return psg_fail(ctx, PSG_E_INVAL, "psg_run_ticks: empty batch");
	if (K >= (1u << 24) || R * K >= (size_t)INT32_MAX)
		return psg_fail(ctx, PSG_E_OVERFLOW, "psg_run_ticks: batch too large");
	PSG_CUDA(cudaSetDevice(ctx->device));
	cudaStream_t st = ctx->stream;
	const size_t nray = R * K;
	ctx->nkev = 0;
	ctx->launches = 0;
	ctx->host_syncs = 0;
	PSG_CUDA(cudaEventRecord(ctx->ev[0], st));
	PsgTraceFill tf;
	int rc = psg_trace_fill(ctx, d_rays, nray, &tf);
	if (rc) return rc;
	BatchPlan pl;
	rc = plan_batch(ctx, R, K, tf, pl);
	if (rc) return rc;
	PSG_CUDA(cudaEventRecord(ctx->ev[1], st));
	k_set_batch<<<1, 1, 0, st>>>(ctx->d_batch, first_tick, tick_time, d_rays, d_rays);
	PSG_CHECK_LAUNCH();
	ctx->launches++;
	PSG_CUDA(cudaMemsetAsync(ctx->d_counters + 1, 0, 2 * sizeof(unsigned long long), st));
	PSG_CUDA(cudaMemsetAsync(ctx->d_counters + 6, 0, sizeof(unsigned long long), st));
	// per-launch timing needs the launches issued one by one
	const bool graph = ctx->use_graphs && !ctx->timing;
	rc = graph ? launch_graph(ctx, batch_key(ctx, pl, ctx->d_batch), [&] { return enqueue_any(ctx, pl, ctx->d_batch); })
			: enqueue_any(ctx, pl, ctx->d_batch);
	if (rc) return rc;
	PSG_CUDA(cudaEventRecord(ctx->ev[2], st));
	// the batch's counters and status, one synchronisation
	unsigned long long cnt[9];
	uint32_t stw = 0;
	PSG_CUDA(cudaMemcpyAsync(cnt, ctx->d_counters, sizeof(cnt), cudaMemcpyDeviceToHost, st));
	PSG_CUDA(cudaMemcpyAsync(&stw, ctx->d_status, sizeof(stw), cudaMemcpyDeviceToHost, st));
	PSG_CUDA(cudaStreamSynchronize(st));
	ctx->host_syncs++;
	if (stw) {
		PSG_CUDA(cudaMemsetAsync(ctx->d_status, 0, sizeof(uint32_t), st));
		return psg_fail(ctx, PSG_E_DEVICE, "device status 0x%x:%s%s%s", stw,
				(stw & PSG_ST_NAN) ? " non-finite state" : "",
				(stw & PSG_ST_SOLVER) ? " integrator step limit" : "",
				(stw & PSG_ST_IE_NEG) ? " negative internal energy" : "");
	}
	const unsigned long long nsat = cnt[1];
	ctx->sat_frac = tf.nhit ? (double)nsat / (double)tf.nhit : 0.0;
	if (stats) {
		double lost = 0.0;
		memcpy(&lost, &cnt[2], sizeof(double));
		float trace_ms = 0.f, tick_ms = 0.f;
		cudaEventElapsedTime(&trace_ms, ctx->ev[0], ctx->ev[1]);
		cudaEventElapsedTime(&tick_ms, ctx->ev[1], ctx->ev[2]);
		stats->hits = (double)tf.nhit;
		stats->saturated = (double)nsat;
		stats->active = (double)cnt[6];
		stats->lost_photons = lost;
		stats->trace_ms = trace_ms;
		stats->tick_ms = tick_ms;
		stats->launches = (double)ctx->launches;
		stats->surrogate_accepted = pl.surr ? (double)cnt[8] : 0.0;
		stats->rec_rays = stats->rec_photons = 0.0;
		stats->host_syncs = (double)ctx->host_syncs;
		for (int k = 0; k < PSG_K_NKERNELS; k++) stats->kernel_ms[k] = stats->kernel_launches[k] = 0.0;
		for (int i = 0; i < ctx->nkev; i++) {
			float ms = 0.f;
			cudaEventElapsedTime(&ms, ctx->kev[2 * i], ctx->kev[2 * i + 1]);
			stats->kernel_ms[ctx->kev_kind[i]] += ms;
			stats->kernel_launches[ctx->kev_kind[i]] += 1.0;
		}
	}
	return PSG_OK;
}

extern "C" int psg_run_ticks_device(psg_context *ctx, const psg_ray *d_rays, size_t R, size_t K,
		int64_t first_tick, double tick_time, psg_tick_stats *stats) {
	if (!ctx) return PSG_E_INVAL;
	if (!ctx->have_physics || !ctx->have_tree)
		return psg_fail(ctx, PSG_E_INVAL, "psg_run_ticks: set physics, load particles and build the tree first");
	if (R == 0 || K == 0 || !d_rays) return psg_fail(ctx, PSG_E_INVAL, "psg_run_ticks: empty batch");
	if (!ctx->flags.on_the_spot) {
		PSG_CUDA(cudaSetDevice(ctx->device));
		return psg_run_ticks_rec(ctx, d_rays, R, K, first_tick, tick_time, stats);
	}
	return psg_run_ticks_core(ctx, d_rays, R, K, first_tick, tick_time, stats);
}

int psg_run_ticks_rec_graph(psg_context *ctx, const psg_ray *d_rays, size_t R, size_t K, int64_t first_tick,
		double tick_time, psg_tick_stats *stats) {
	if (!ctx->have_physics || !ctx->have_tree) return PSG_RETRY;
	const int nspec = ctx->flags.h_only ? 1 : 3;
	const size_t cap_rec = (size_t)ctx->rec_nrec * nspec;
	const size_t nray = R + cap_rec;
	// the slabs and hit buffers as an earlier call left them: the first call
	// runs its ticks one by one, which sizes them
	if (ctx->rec_nrec <= 0 || !ctx->slab_cap || !ctx->batch_cap ||
			nray >= (size_t)INT32_MAX)
		return PSG_RETRY;
	PSG_CUDA(cudaSetDevice(ctx->device));
	cudaStream_t st = ctx->stream;
	ctx->nkev = 0;
	ctx->launches = 0;
	ctx->host_syncs = 0;
	psg_ray *buf = (psg_ray *)psg_scratch(ctx, S_RECRAYS, sizeof(psg_ray) * nray);
	if (!buf) return PSG_E_NOMEM;
	// the call's source rays do not depend on the ticks' updates: traced and
	// sorted together first (one host wait), each tick traverses only the
	// rays it emits
	int rc = psg_trace_src_batch(ctx, d_rays, R * K);
	if (rc) return rc;
	rc = psg_trace_fill_prepare(ctx, nray);
	if (!rc) rc = psg_rec_prepare(ctx);
	if (rc) return rc;
	PsgTraceFill tf{ctx->batch_cap, ctx->slab_cap, ctx->slab_cap};
	BatchPlan pl;
	pl.src_R = R;
	rc = plan_batch(ctx, nray, 1, tf, pl);
	if (rc) return rc;
	rc = psg_state_save(ctx);      // (the undo if a tick outgrows the buffers)
	if (rc) return rc;
	PsgBatchDev *B = ctx->d_batch;
	k_set_batch<<<1, 1, 0, st>>>(B, first_tick, tick_time, buf, d_rays);
	PSG_CHECK_LAUNCH();
	unsigned long long *cnt = ctx->d_counters;
	PSG_CUDA(cudaMemsetAsync(cnt + 1, 0, 3 * sizeof(unsigned long long), st));      // 1-3
	PSG_CUDA(cudaMemsetAsync(cnt + 6, 0, 2 * sizeof(unsigned long long), st));      // 6, 7
	PSG_CUDA(cudaMemsetAsync(cnt + 10, 0, sizeof(unsigned long long), st));
	PSG_CUDA(cudaMemsetAsync(cnt + 14, 0, sizeof(unsigned long long), st));
	PSG_CUDA(cudaMemsetAsync(cnt + 24, 0, sizeof(unsigned long long), st));
	const int64_t *off64 = (const int64_t *)ctx->scratch[S_OFFSETS].p;
	const unsigned *nlim = (const unsigned *)(cnt + 15);
	auto tick_enqueue = [&]() -> int {
		k_rec_src<<<(unsigned)std::min<size_t>(blocks(R, 256), 4 * (size_t)ctx->sms), 256, 0, st>>>(B, R, buf);
		PSG_CHECK_LAUNCH();
		int r = psg_rec_emit_enqueue(ctx, B, buf + R, cnt + 15, cnt + 14);
		if (r) return r;
		r = psg_trace_rec_fill_enqueue(ctx, buf, R, cap_rec, nlim, pl.cap, B);
		if (r) return r;
		r = enqueue_any(ctx, pl, B);
		if (r) return r;
		r = psg_rec_mark_enqueue(ctx, R, B);
		if (r) return r;
		k_rec_tick_end<<<1, 1, 0, st>>>(off64, nray, cnt + 7, B);
		PSG_CHECK_LAUNCH();
		ctx->launches += 3;
		return PSG_OK;
	};
	std::vector<unsigned long long> key = batch_key(ctx, pl, B);
	key.push_back(0x5245432d5449434bull);      // a recombination tick
	key.push_back(R);
	key.push_back(cap_rec);
	key.push_back((unsigned long long)(uintptr_t)buf);
	key.push_back((unsigned long long)(uintptr_t)ctx->d_lte);
	key.push_back(ctx->rec_seed);
	key.push_back((unsigned long long)ctx->rec_disable_lte);
	key.push_back((unsigned long long)(uintptr_t)ctx->d_srcmark);
	key.push_back(ctx->trace_grid);
	key.push_back((unsigned long long)ctx->tune.trace_warps);
	rc = launch_graph(ctx, std::move(key), tick_enqueue, K);
	if (rc) return rc;
	unsigned long long c[32];
	uint32_t stw = 0;
	PSG_CUDA(cudaMemcpyAsync(c, cnt, sizeof(c), cudaMemcpyDeviceToHost, st));
	PSG_CUDA(cudaMemcpyAsync(&stw, ctx->d_status, sizeof(stw), cudaMemcpyDeviceToHost, st));
	PSG_CUDA(cudaStreamSynchronize(st));
	ctx->host_syncs++;
	if (stw & PSG_ST_SLAB) {
		// a tick outgrew the slabs or the hit buffers: undo the call, size
		// both for what was seen, and let the ticks run one by one
		PSG_CUDA(cudaMemsetAsync(ctx->d_status, 0, sizeof(uint32_t), st));
		rc = psg_state_restore(ctx);
		if (rc) return rc;
		if (c[3] > ctx->slab_cap) {
			size_t want = 1024;
			while (want < c[3] + c[3] / 4) want <<= 1;
			ctx->slab_cap = want;
		}
		if (c[24] > ctx->batch_cap) ctx->batch_cap = ((size_t)(c[24] + c[24] / 8) + 65535) & ~(size_t)65535;
		return PSG_RETRY;
	}
	if (stw) {
		PSG_CUDA(cudaMemsetAsync(ctx->d_status, 0, sizeof(uint32_t), st));
		return psg_fail(ctx, PSG_E_DEVICE, "device status 0x%x:%s%s%s", stw,
				(stw & PSG_ST_NAN) ? " non-finite state" : "",
				(stw & PSG_ST_SOLVER) ? " integrator step limit" : "",
				(stw & PSG_ST_IE_NEG) ? " negative internal energy" : "");
	}
	const unsigned *last = (const unsigned *)&c[11];
	ctx->rec_last = (size_t)last[0] + last[1] + last[2];
	ctx->rec_last_R = R;
	ctx->rec_last_kmax = cap_rec;
	ctx->rec_last_threshold = ctx->rec_nrec < 0;
	ctx->sat_frac = c[7] ? (double)c[1] / (double)c[7] : 0.0;
	if (stats) {
		memset(stats, 0, sizeof(*stats));
		stats->hits = (double)c[7];
		stats->saturated = (double)c[1];
		stats->active = (double)c[6];
		memcpy(&stats->lost_photons, &c[2], sizeof(double));
		stats->launches = (double)ctx->launches;
		stats->rec_rays = (double)c[14];
		memcpy(&stats->rec_photons, &c[10], sizeof(double));
		stats->host_syncs = (double)ctx->host_syncs;
	}
	return PSG_OK;
}

// ---- the autotuner -------------------------------------------------------------
extern "C" int psg_autotune(psg_context *ctx, const psg_ray *d_rays, size_t R, size_t K, int64_t first_tick,
		double tick_time, int reps, psg_tune *out, double *best_ms) {
	if (!ctx) return PSG_E_INVAL;
	if (!d_rays || R == 0 || K == 0) return psg_fail(ctx, PSG_E_INVAL, "psg_autotune: empty batch");
	if (!ctx->have_physics || !ctx->have_tree)
		return psg_fail(ctx, PSG_E_INVAL, "psg_autotune: set physics, load particles and build the tree first");
	if (reps < 1) reps = 1;
	PSG_CUDA(cudaSetDevice(ctx->device));
	const int timing0 = ctx->timing;
	ctx->timing = 0;
	const double sat0 = ctx->sat_frac;
	int rc = psg_state_save(ctx);
	if (rc) return rc;
	// one shape: a warm-up batch (it captures the shape's graph), then reps
	// timed batches; the state goes back after every one
	auto trial = [&](const psg_tune &t, double *ms) -> int {
		ctx->tune = t;
		double best = 1e300;
		for (int r = 0; r <= reps; r++) {
			PSG_CUDA(cudaEventRecord(ctx->ev[5], ctx->stream));
			const int rc1 = psg_run_ticks_device(ctx, d_rays, R, K, first_tick, tick_time, nullptr);
			PSG_CUDA(cudaEventRecord(ctx->ev[6], ctx->stream));
			PSG_CUDA(cudaEventSynchronize(ctx->ev[6]));
			const int rc2 = psg_state_restore(ctx);
			ctx->sat_frac = sat0;
			if (rc1) return rc1;
			if (rc2) return rc2;
			float e = 0.f;
			PSG_CUDA(cudaEventElapsedTime(&e, ctx->ev[5], ctx->ev[6]));
			if (r > 0) best = std::min(best, (double)e);
		}
		*ms = best;
		return PSG_OK;
	};
	psg_tune cur = ctx->tune;
	double cur_ms = 0.0;
	rc = trial(cur, &cur_ms);
	// a candidate is kept when it is at least 1% faster (timing noise)
	auto consider = [&](const psg_tune &t) -> int {
		double ms = 0.0;
		const int r = trial(t, &ms);
		if (r) return r;
		if (ms < 0.99 * cur_ms) {
			cur = t;
			cur_ms = ms;
		}
		return PSG_OK;
	};
	// traversal warps per block (the packet: one ray per warp, warps per block)
	const int warps[] = {2, 4, 8};
	for (int w : warps) {
		if (rc || w == cur.trace_warps) continue;
		psg_tune t = cur;
		t.trace_warps = w;
		rc = consider(t);
	}
	// deposit groups: which rays take a warp, a 128-thread group, a block
	const int thr[][2] = {{64, 256}, {96, 384}, {128, 512}, {192, 768}, {256, 1024}, {384, 1536}, {512, 2048},
			{768, 3072}};
	for (auto &th : thr) {
		if (rc || (th[0] == cur.deposit_long && th[1] == cur.deposit_mid)) continue;
		psg_tune t = cur;
		t.deposit_long = th[0];
		t.deposit_mid = th[1];
		rc = consider(t);
	}
	// the integrator's registers (occupancy against spills)
	for (int mb : {1, 3, 4}) {
		if (rc || mb == cur.update_minblocks) continue;
		psg_tune t = cur;
		t.update_minblocks = mb;
		rc = consider(t);
	}
	// which runs are sorted before their sums, which put in order where summed
	for (int rs : {4, 8, 16}) {
		if (rc || rs == cur.run_short) continue;
		psg_tune t = cur;
		t.run_short = rs;
		rc = consider(t);
	}
	// the order in which the integrator claims the particles
	for (int uo : {0, 1}) {
		if (rc || uo == cur.update_order) continue;
		psg_tune t = cur;
		t.update_order = uo;
		rc = consider(t);
	}
	ctx->tune = cur;
	ctx->timing = timing0;
	if (rc) return rc;
	psg_tune_store(ctx->device, &cur);
	if (out) *out = cur;
	if (best_ms) *best_ms = cur_ms;
	return PSG_OK;
}

extern "C" int psg_run_ticks(psg_context *ctx, const psg_ray *rays, size_t R, size_t K,
		int64_t first_tick, double tick_time, psg_tick_stats *stats) {
	if (!ctx) return PSG_E_INVAL;
	if (!rays || R == 0 || K == 0) return psg_fail(ctx, PSG_E_INVAL, "psg_run_ticks: empty batch");
	PSG_CUDA(cudaSetDevice(ctx->device));
	psg_ray *d = (psg_ray *)psg_scratch(ctx, S_RAYS, sizeof(psg_ray) * R * K);
	if (!d) return PSG_E_NOMEM;
	PSG_CUDA(cudaMemcpyAsync(d, rays, sizeof(psg_ray) * R * K, cudaMemcpyHostToDevice, ctx->stream));
	return psg_run_ticks_device(ctx, d, R, K, first_tick, tick_time, stats);
}

extern "C" int psg_step_evolve(psg_context *ctx, psg_step *steps, size_t n) {
	if (!ctx) return PSG_E_INVAL;
	if (!ctx->have_physics) return psg_fail(ctx, PSG_E_INVAL, "psg_step_evolve: set physics first");
	if (n == 0) return PSG_OK;
	if (!steps) return psg_fail(ctx, PSG_E_INVAL, "psg_step_evolve: null steps");
	PSG_CUDA(cudaSetDevice(ctx->device));
	psg_step *d = (psg_step *)psg_scratch(ctx, S_MISC, sizeof(psg_step) * n);
	if (!d) return PSG_E_NOMEM;
	cudaStream_t st = ctx->stream;
	PSG_CUDA(cudaMemcpyAsync(d, steps, sizeof(psg_step) * n, cudaMemcpyHostToDevice, st));
	k_step_evolve<<<blocks(n, 128), 128, 0, st>>>(d, n, psg_phys_params(ctx), ctx->d_status);
	PSG_CHECK_LAUNCH();
	PSG_CUDA(cudaMemcpyAsync(steps, d, sizeof(psg_step) * n, cudaMemcpyDeviceToHost, st));
	PSG_CUDA(cudaStreamSynchronize(st));
	return check_status(ctx);
}

// ---- step_evolve without allocation -----------------------------------------
// psg_step_evolve_noalloc stages the steps in a fixed buffer that is part of
// the library's device image instead of the context's growable scratch, so
// the call itself never allocates or frees device memory. It is meant for
// hosts that cannot allocate while a time step is under way: a code whose
// own pool allocator has already taken the device's free memory (cudaMalloc
// would fail there), or one that must not pay the device-wide
// synchronisation that cudaMalloc and cudaFree can imply while its other
// streams are busy. The buffer holds PSG_NOALLOC_MAX_STEPS steps (2.25 MiB)
// plus a status word; every device gets its own copy, held until the process
// exits. There is one buffer per device, not per context: calls that overlap
// in time on the same device (two host threads, two contexts or two streams)
// race on it, and the caller must serialise them.
static constexpr size_t kNoallocStatusOffset = (size_t)PSG_NOALLOC_MAX_STEPS * sizeof(psg_step);
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocStatusOffset + 256];

// Device address of the static buffer on the current device. The lookup
// loads this file's module on that device if it is not loaded yet (CUDA
// loads modules lazily), and loading the module is what reserves the
// buffer: psg_create() calls this once so that the reservation happens when
// the context is made, before a host's pool allocator takes the device's
// free memory. Each psg_step_evolve_noalloc() call looks the address up
// again rather than caching it, so a host that reset the device in between
// gets the buffer of the new primary context, not a stale address.
int psg_noalloc_lookup(unsigned char **base) {
	void *p = nullptr;
	const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
	if (e != cudaSuccess || !p) {
		cudaGetLastError();
		return e != cudaSuccess ? (int)e : (int)cudaErrorInvalidSymbol;
	}
	*base = (unsigned char *)p;
	return 0;
}

extern "C" int psg_step_evolve_noalloc(psg_context *ctx, psg_step *steps, size_t n) {
	if (!ctx) return PSG_E_INVAL;
	if (!ctx->have_physics) return psg_fail(ctx, PSG_E_INVAL, "psg_step_evolve_noalloc: set physics first");
	if (n > PSG_NOALLOC_MAX_STEPS)
		return psg_fail(ctx, PSG_E_INVAL,
				"psg_step_evolve_noalloc: %zu steps exceed its fixed buffer of %d; split the call or use "
				"psg_step_evolve", n, PSG_NOALLOC_MAX_STEPS);
	if (n == 0) return PSG_OK;
	if (!steps) return psg_fail(ctx, PSG_E_INVAL, "psg_step_evolve_noalloc: null steps");
	PSG_CUDA(cudaSetDevice(ctx->device));
	unsigned char *base = nullptr;
	const int e = psg_noalloc_lookup(&base);
	if (e) return psg_cuda_fail(ctx, (cudaError_t)e, "cudaGetSymbolAddress(g_noalloc_scratch)", __FILE__, __LINE__);
	psg_step *d = (psg_step *)base;
	uint32_t *d_status = (uint32_t *)(base + kNoallocStatusOffset);
	cudaStream_t st = ctx->stream;
	// the status word is OR-ed into by the kernel: it must start at zero
	PSG_CUDA(cudaMemsetAsync(d_status, 0, sizeof(uint32_t), st));
	PSG_CUDA(cudaMemcpyAsync(d, steps, sizeof(psg_step) * n, cudaMemcpyHostToDevice, st));
	k_step_evolve<<<blocks(n, 128), 128, 0, st>>>(d, n, psg_phys_params(ctx), d_status);
	PSG_CHECK_LAUNCH();
	PSG_CUDA(cudaMemcpyAsync(steps, d, sizeof(psg_step) * n, cudaMemcpyDeviceToHost, st));
	uint32_t status = 0;
	PSG_CUDA(cudaMemcpyAsync(&status, d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
	PSG_CUDA(cudaStreamSynchronize(st));
	if (status)
		return psg_fail(ctx, PSG_E_DEVICE, "device status 0x%x:%s%s%s", status,
				(status & PSG_ST_NAN) ? " non-finite state" : "",
				(status & PSG_ST_SOLVER) ? " integrator step limit" : "",
				(status & PSG_ST_IE_NEG) ? " negative internal energy" : "");
	return PSG_OK;
}

extern "C" int psg_set_update_log(psg_context *ctx, float *d_rows, size_t cap, unsigned long long *d_count) {
	if (!ctx) return PSG_E_INVAL;
	if (d_rows && (!d_count || cap == 0)) return psg_fail(ctx, PSG_E_INVAL, "psg_set_update_log: need a counter and capacity");
	ctx->log_buf = d_rows;
	ctx->log_cap = d_rows ? cap : 0;
	ctx->log_count = d_rows ? d_count : nullptr;
	return PSG_OK;
}
