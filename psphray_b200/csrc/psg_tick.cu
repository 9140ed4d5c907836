// Ticks: deposit (loop.c:388-608), merge (loop.c:610-645) and update
// (loop.c:647-776) for many ticks whose rays are traced in one batch.
//
// Hit lists depend only on geometry, so all rays of a batch of ticks are
// traced together. Before the tick loop every hit gets a slot in a
// by-particle order ((tick, ipar, hit) sorted), which turns the reference's
// merge into the runs of equal (tick, ipar) and its float atomics into a
// fixed-order FP64 sum per particle. Then per tick:
//   deposit: one warp per ray walks its sorted hits 32 at a time; optical
//     depths are summed with an FP64 warp scan, the transmitted photons before
//     each hit are TM*exp(-scan), absorbed = TM_j*(1-e^-tau_j); the first hit
//     whose absorption exceeds its neutral atoms (the cap of loop.c:482-485)
//     or after which TM/Nph < 1e-10 (loop.c:585) is settled on its own and the
//     scan restarts after it. Each hit writes photons/NH into its slot, or -1
//     when the reference would not deposit there;
//   update: one thread per particle hit in the tick sums its slots in order
//     and advances (lambdaH, ie) by the step since its last hit.
#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "psg_internal.cuh"
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


// (tick, ipar) keys for the by-particle order, tick in the bits above
// `shift`; one warp per ray. KT is 32-bit whenever both fit.
template <typename KT>
__global__ void k_slot_keys(size_t nray, int nray_per_tick, int shift, const int64_t *__restrict__ off,
		const uint32_t *__restrict__ ipar, KT *__restrict__ keys, uint32_t *__restrict__ vals) {
	const size_t r = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) / 32;
	const int lane = threadIdx.x & 31;
	if (r >= nray) return;
	const KT t = (KT)(r / (size_t)nray_per_tick);
	for (int64_t h = off[r] + lane; h < off[r + 1]; h += 32) {
		keys[h] = (t << shift) | (KT)ipar[h];
		vals[h] = (uint32_t)h;
	}
}

template <typename KT>
__global__ void k_slots(size_t nhit, const KT *__restrict__ skeys, const uint32_t *__restrict__ svals,
		uint32_t *__restrict__ slot, int32_t *__restrict__ head) {
	const size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
	if (k >= nhit) return;
	slot[svals[k]] = (uint32_t)k;
	head[k] = (k == 0 || skeys[k] != skeys[k - 1]) ? 1 : 0;
}

template <typename KT>
__global__ void k_active(size_t nhit, int shift, const KT *__restrict__ skeys, const int32_t *__restrict__ head,
		const int32_t *__restrict__ scan, uint32_t *__restrict__ act_ipar, uint32_t *__restrict__ act_seg,
		KT *__restrict__ act_key) {
	const size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
	if (k >= nhit) return;
	if (!head[k]) return;
	const int a = scan[k];
	act_ipar[a] = (uint32_t)(skeys[k] & (((KT)1 << shift) - 1));
	act_seg[a] = (uint32_t)k;
	act_key[a] = skeys[k];
}

// first active entry of every tick (and the total at index nticks)
template <typename KT>
__global__ void k_tick_bounds(int nticks, int shift, const KT *__restrict__ act_key, int nact,
		uint32_t *__restrict__ act_seg, uint32_t nhit, int32_t *__restrict__ tick_act) {
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t > nticks) return;
	int lo = 0, hi = nact;
	if (t < nticks) {
		const KT want = (KT)t << shift;
		while (lo < hi) {
			const int mid = (lo + hi) / 2;
			if (act_key[mid] < want) lo = mid + 1; else hi = mid;
		}
	} else {
		lo = nact;
	}
	tick_act[t] = lo;
	if (t == nticks) act_seg[nact] = nhit;
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
// as loop.c:580 updates TM. Each hit writes photons/NH to its slot, or -1
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

// One hit's deposits sit together, nacc doubles per slot (photons/NH; with
// heat the heat; with helium yGdepHeI and yGdepHeII), so that the scattered
// store of a hit touches one 32-byte sector and the by-particle sums read
// one contiguous run.
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
		const uint32_t *__restrict__ hipar, const double *__restrict__ hkern, const uint32_t *__restrict__ slot,
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
	uint32_t np_slot = 0;
	double np_kern = 0.0, np_lam = 0.0;
	float np_mass = 1.0f;
	{
		const int64_t h = h0 + t;
		if (h < h1) {
			const uint32_t p = hipar[h];
			np_kern = hkern[h];
			np_slot = slot[h];
			if (!done) { np_lam = lambdaH[p]; np_mass = mass[p]; }
		}
	}
	for (int64_t base = h0; base < h1; base += NT) {
		const int64_t h = base + t;
		const bool valid = h < h1;
		const double kern_c = np_kern, lam_c = np_lam;
		const float mass_c = np_mass;
		const uint32_t slot_c = np_slot;
		{
			const int64_t hn = h + NT;
			if (hn < h1) {
				const uint32_t p = hipar[hn];
				np_kern = hkern[hn];
				np_slot = slot[hn];
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
// increments (nacc of them per slot), with the secondary
// ionisation and heating of loop.c:513-552 (whose HeII terms the
// reference's statements drop, loop.c:523,542).
template <int NT>
__device__ void deposit_ray_gen(const psg_ray &ray, int64_t h0, int64_t h1, int t,
		const uint32_t *__restrict__ hipar, const double *__restrict__ hkern, const uint32_t *__restrict__ slot,
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
	uint32_t np_slot = 0;
	double np_kern = 0.0, np_lam = 0.0, np_l1 = 0.0, np_l2 = 0.0;
	float np_mass = 1.0f;
	{
		const int64_t h = h0 + t;
		if (h < h1) {
			const uint32_t p = hipar[h];
			np_kern = hkern[h];
			np_slot = slot[h];
			if (!done) { np_lam = lambdaH[p]; np_mass = mass[p]; np_l1 = P.lamHeI[p]; np_l2 = P.lamHeII[p]; }
		}
	}
	for (int64_t base = h0; base < h1; base += NT) {
		const int64_t h = base + t;
		const bool valid = h < h1;
		const double kern_c = np_kern, lam_c = np_lam, l1_c = np_l1, l2_c = np_l2;
		const float mass_c = np_mass;
		const uint32_t slot_c = np_slot;
		{
			const int64_t hn = h + NT;
			if (hn < h1) {
				const uint32_t p = hipar[hn];
				np_kern = hkern[hn];
				np_slot = slot[hn];
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

// Blocks [0, nlong) take one long ray each with all DEP_THREADS threads;
// the next nmid_blocks take four middle rays each, 128 threads per ray; the
// remaining blocks take DEP_THREADS/32 short rays, one per warp.
#define DEP_THREADS 512
#define DEP_LONG 96       // more hits than this: a group of threads, else a warp
#define DEP_MID 384       // more hits than this: the whole block, else a 128-thread quarter

template <bool GEN, bool AFF>
__global__ void __launch_bounds__(DEP_THREADS, 2) k_deposit(const psg_ray *__restrict__ rays,
		const uint32_t *__restrict__ long_rays, int nlong, const uint32_t *__restrict__ mid_rays, int nmid,
		const uint32_t *__restrict__ short_rays, int nshort,
		const int64_t *__restrict__ off, const uint32_t *__restrict__ hipar, const double *__restrict__ hkern,
		const uint32_t *__restrict__ slot, const double *__restrict__ lambdaH, const float *__restrict__ mass,
		PhysParams P, int want_heat, double *__restrict__ acc, int nacc, unsigned long long *__restrict__ n_sat,
		double *__restrict__ lost) {
	__shared__ DepShared sh_block;
	__shared__ DepShared sh_quarter[4];
	__shared__ DepShared sh_warp[DEP_THREADS / 32];
	const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
	unsigned nsat = 0;
	double tm_lost = 0.0;
	const int nmid_blocks = (nmid + 3) / 4;
	if ((int)blockIdx.x < nlong) {
		const uint32_t r = long_rays[blockIdx.x];
		if (GEN)
			deposit_ray_gen<DEP_THREADS>(rays[r], off[r], off[r + 1], tid, hipar, hkern, slot, lambdaH, mass, P,
					want_heat, acc, nacc, sh_block, nsat, tm_lost, 0);
		else
			deposit_ray<DEP_THREADS, AFF>(rays[r], off[r], off[r + 1], tid, hipar, hkern, slot, lambdaH, mass, P,
					want_heat, acc, sh_block, nsat, tm_lost, 0);
	} else if ((int)blockIdx.x < nlong + nmid_blocks) {
		const int q = tid >> 7;
		const int m = ((int)blockIdx.x - nlong) * 4 + q;
		if (m < nmid) {
			const uint32_t r = mid_rays[m];
			if (GEN)
				deposit_ray_gen<128>(rays[r], off[r], off[r + 1], tid & 127, hipar, hkern, slot, lambdaH, mass, P,
						want_heat, acc, nacc, sh_quarter[q], nsat, tm_lost, 1 + q);
			else
				deposit_ray<128, AFF>(rays[r], off[r], off[r + 1], tid & 127, hipar, hkern, slot, lambdaH, mass, P,
						want_heat, acc, sh_quarter[q], nsat, tm_lost, 1 + q);
		}
	} else {
		const int w = ((int)blockIdx.x - nlong - nmid_blocks) * (DEP_THREADS / 32) + wid;
		if (w < nshort) {
			const uint32_t r = short_rays[w];
			if (off[r + 1] > off[r]) {
				if (GEN)
					deposit_ray_gen<32>(rays[r], off[r], off[r + 1], lane, hipar, hkern, slot, lambdaH, mass, P,
							want_heat, acc, nacc, sh_warp[wid], nsat, tm_lost, 0);
				else
					deposit_ray<32, AFF>(rays[r], off[r], off[r + 1], lane, hipar, hkern, slot, lambdaH, mass, P,
							want_heat, acc, sh_warp[wid], nsat, tm_lost, 0);
			}
		}
	}
	for (int o = 16; o > 0; o >>= 1) nsat += __shfl_down_sync(0xffffffffu, nsat, o);
	if (lane == 0 && nsat) atomicAdd(n_sat, (unsigned long long)nsat);
	if (lane == 0 && tm_lost != 0.0) atomicAdd(lost, tm_lost);
}

// Rays of the batch split into long, middle and short lists (ray order
// kept): cls = 1 for long, 1 << 32 for middle, so one scan counts both.
__global__ void k_ray_class(size_t nray, const int64_t *__restrict__ off, unsigned long long *__restrict__ cls) {
	const size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
	if (r >= nray) return;
	const int64_t n = off[r + 1] - off[r];
	cls[r] = n > DEP_MID ? 1ull : (n > DEP_LONG ? (1ull << 32) : 0ull);
}

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
__global__ void k_act_class(size_t na, const uint32_t *__restrict__ act_seg, int32_t *__restrict__ flag) {
	const size_t a = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
	if (a > na) return;
	flag[a] = (a < na && act_seg[a + 1] - act_seg[a] > 32) ? 1 : 0;
}
__global__ void k_act_lists(size_t na, const int32_t *__restrict__ flag, const int32_t *__restrict__ scan,
		uint32_t *__restrict__ long_act) {
	const size_t a = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
	if (a < na && flag[a]) long_act[scan[a]] = (uint32_t)a;
}
// first long entry of every tick
__global__ void k_tick_long(int K, const int32_t *__restrict__ tick_act, const int32_t *__restrict__ scan,
		int32_t *__restrict__ out) {
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t <= K) out[t] = scan[tick_act[t]];
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

// The particle's summed deposits of the tick: isothermal, the closed-form
// update_pars() step (loop.c:653-770); otherwise the sums for the integrator.
template <bool ISO, bool REC>
__device__ __forceinline__ void finish_particle(int a, double g, double heat, int nh,
		const uint32_t *__restrict__ act_ipar, int32_t *__restrict__ hits, double *__restrict__ act_g,
		double *__restrict__ act_heat, double *__restrict__ lambdaH, float *__restrict__ ie,
		int64_t *__restrict__ lasthit, const float *__restrict__ rho, const float *__restrict__ yeMET,
		const float *__restrict__ hstep, UpdRec *__restrict__ rec, int lo, const double *__restrict__ gcarry,
		const PhysParams &P, int64_t tick, double tick_time, uint32_t *__restrict__ status) {
	const uint32_t p = act_ipar[a];
	hits[p] += nh;
	if (gcarry) g += gcarry[p];      // photons left over by an earlier explicit step (loop.c:745)
	if (!ISO) {
		if (act_g) {        // read by the surrogate and the update log only
			act_g[a] = g;
			act_heat[a] = heat;
		}
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

// Per-particle sums of one tick's deposits (photons/NH, heat, deposit count)
// in slot order. The first long_blocks blocks take the tick's long segments,
// a warp each: lanes strided over the segment (eight loads in flight per
// lane), then a fixed butterfly. The other blocks take the short ones, a
// thread each. Particles are in leaf order, so the long ones are neighbours;
// giving each its own warp keeps them from piling up on a few warps.
template <bool ISO, bool REC>
__global__ void __launch_bounds__(256) k_reduce(int t, const int32_t *__restrict__ tick_act,
		const uint32_t *__restrict__ act_ipar, const uint32_t *__restrict__ act_seg,
		const double *__restrict__ acc, int want_heat,
		const uint32_t *__restrict__ long_act, int nlong, int long_blocks,
		int32_t *__restrict__ hits, double *__restrict__ act_g, double *__restrict__ act_heat,
		double *__restrict__ lambdaH, float *__restrict__ ie, int64_t *__restrict__ lasthit,
		const float *__restrict__ rho, const float *__restrict__ yeMET, const float *__restrict__ hstep,
		UpdRec *__restrict__ rec, const double *__restrict__ gcarry, PhysParams P, int64_t tick, double tick_time,
		uint32_t *__restrict__ status) {
	if ((int)blockIdx.x < long_blocks) {
		const int e = blockIdx.x * 8 + (threadIdx.x >> 5);
		const int lane = threadIdx.x & 31;
		if (e >= nlong) return;
		const int a = (int)long_act[e];
		const uint32_t b0 = act_seg[a], b1 = act_seg[a + 1];
		double sg = 0.0, sh = 0.0;
		int sn = 0;
		uint32_t k = b0 + lane;
		if (want_heat) {
			const double2 *acc2 = reinterpret_cast<const double2 *>(acc);
			for (; k + 7 * 32 < b1; k += 8 * 32) {
				double2 v[8];
#pragma unroll
				for (int u = 0; u < 8; u++) v[u] = acc2[k + 32 * u];
#pragma unroll
				for (int u = 0; u < 8; u++)
					if (v[u].x >= 0.0) { sg += v[u].x; sh += v[u].y; sn++; }
			}
			for (; k < b1; k += 32) {
				const double2 d = acc2[k];
				if (d.x >= 0.0) { sg += d.x; sh += d.y; sn++; }
			}
		} else {
			for (; k + 7 * 32 < b1; k += 8 * 32) {
				double v[8];
#pragma unroll
				for (int u = 0; u < 8; u++) v[u] = acc[k + 32 * u];
#pragma unroll
				for (int u = 0; u < 8; u++)
					if (v[u] >= 0.0) { sg += v[u]; sn++; }
			}
			for (; k < b1; k += 32) {
				const double d = acc[k];
				if (d >= 0.0) { sg += d; sn++; }
			}
		}
#pragma unroll
		for (int o = 16; o > 0; o >>= 1) {
			sg += __shfl_xor_sync(0xffffffffu, sg, o);
			sh += __shfl_xor_sync(0xffffffffu, sh, o);
			sn += __shfl_xor_sync(0xffffffffu, sn, o);
		}
		if (lane == 0)
			finish_particle<ISO, REC>(a, sg, sh, sn, act_ipar, hits, act_g, act_heat, lambdaH, ie, lasthit, rho, yeMET,
					hstep, rec, tick_act[t], gcarry, P, tick, tick_time, status);
		return;
	}
	const int a = tick_act[t] + (blockIdx.x - long_blocks) * blockDim.x + threadIdx.x;
	if (a >= tick_act[t + 1]) return;
	const uint32_t s0 = act_seg[a], s1 = act_seg[a + 1];
	if (s1 - s0 > 32) return;
	double g = 0.0, heat = 0.0;
	int nh = 0;
	for (uint32_t k = s0; k < s1; k++) {
		if (want_heat) {
			const double2 d = reinterpret_cast<const double2 *>(acc)[k];
			if (d.x >= 0.0) { g += d.x; heat += d.y; nh++; }
		} else {
			const double d = acc[k];
			if (d >= 0.0) { g += d; nh++; }
		}
	}
	finish_particle<ISO, REC>(a, g, heat, nh, act_ipar, hits, act_g, act_heat, lambdaH, ie, lasthit, rho, yeMET, hstep,
			rec, tick_act[t], gcarry, P, tick, tick_time, status);
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
__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gmem_src) {
	asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(smem_dst)),
			"l"(gmem_src)
			: "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

#define UPD_WARPS 8
// Every warp owns two buffers of 32 records in shared memory: it claims
// chunks of 32 particles from the tick's cursor and copies their records
// with cp.async one chunk ahead, so a lane whose particle is done takes the
// next one from shared memory without waiting on a gather.
template <bool REC>
__global__ void __launch_bounds__(32 * UPD_WARPS) k_update_queue(int t, const int32_t *__restrict__ tick_act,
		const UpdRec *__restrict__ rec, double *__restrict__ lambdaH, float *__restrict__ ie,
		int64_t *__restrict__ lasthit, float *__restrict__ hstep, PhysParams P, int64_t tick,
		unsigned *__restrict__ cursor, StiffItem *__restrict__ stiff, unsigned *__restrict__ nstiff,
		const uint32_t *__restrict__ alist, const unsigned *__restrict__ nalist, uint32_t *__restrict__ status) {
	__shared__ UpdRec buf[UPD_WARPS][2][32];
	// the tick's particles, or only those listed in alist (the surrogate's rejects)
	const int lo = tick_act[t], hi = tick_act[t + 1];
	const unsigned n = alist ? *nalist : (unsigned)(hi - lo);
	const int lane = threadIdx.x & 31;
	const unsigned lt_mask = (1u << lane) - 1u;
	UpdRec (*B)[32] = buf[threadIdx.x >> 5];
	auto fetch = [&](int b) -> int {
		unsigned base = 0;
		if (lane == 0) base = atomicAdd(cursor, 32u);
		base = __shfl_sync(0xffffffffu, base, 0);
		const int cnt = base >= n ? 0 : (int)min(32u, n - base);
		if (lane < cnt) {
			const unsigned k = base + lane;
			const int a = alist ? (int)alist[k] : lo + (int)k;
			const char *src = (const char *)(rec + (a - lo));
			char *dst = (char *)&B[b][lane];
#pragma unroll
			for (int q = 0; q < 5; q++) cp_async16(dst + 16 * q, src + 16 * q);
		}
		cp_async_commit();
		return cnt;
	};
	int avail[2];
	avail[0] = fetch(0);
	avail[1] = fetch(1);
	cp_async_wait<1>();
	__syncwarp();
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
				cp_async_wait<0>();
				__syncwarp();
				cur ^= 1;
				used = 0;
				avail[cur ^ 1] = fetch(cur ^ 1);
				continue;
			}
			const int rank = __popc(need & lt_mask);
			const int take = min(__popc(need), left);
			if (!have && rank < take) {
				const UpdRec &r = B[cur][used + rank];
				p = r.p;
				const double ie0 = (double)r.ie0;
				const double T = ieye2T(P, ie0, rn_dadd(rn_dsub(1.0, r.lam0), P.he_e));
				cx = make_rhs_ctx(P, (double)r.yeMET, r.g, r.heat, r.time, rn_dmul(P.H_PER_MASS, (double)r.rho), T);
				S.x[0] = r.lam0;
				S.x[1] = ie0;
				S.k1[0] = r.k0;
				S.k1[1] = r.k1;
				S.rec = 0.0;
				S.krec = r.krec;
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
	cp_async_wait<0>();
	if (st) atomicOr(status, st);
}

// The stiff particles of a tick, one thread each (their number is read on
// the device): Rosenbrock from where the explicit steps stopped.
template <bool REC>
__global__ void __launch_bounds__(64) k_update_stiff(const StiffItem *__restrict__ stiff,
		const unsigned *__restrict__ nstiff, double *__restrict__ lambdaH, float *__restrict__ ie,
		int64_t *__restrict__ lasthit, PhysParams P, int64_t tick, uint32_t *__restrict__ status) {
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
		int64_t *__restrict__ lasthit, double *__restrict__ gcarry, PhysParams P, int64_t tick,
		uint32_t *__restrict__ status) {
	const int lo = tick_act[t];
	const int a = lo + blockIdx.x * blockDim.x + threadIdx.x;
	if (a >= tick_act[t + 1]) return;
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

template <bool REC>
__global__ void __launch_bounds__(128, 4) k_update_he(int t, const int32_t *__restrict__ tick_act,
		const uint32_t *__restrict__ act_ipar, const uint32_t *__restrict__ act_seg, const double *__restrict__ acc,
		int want_heat,
		int32_t *__restrict__ hits, double *__restrict__ lambdaH, float *__restrict__ ie,
		int64_t *__restrict__ lasthit, const float *__restrict__ rho, const float *__restrict__ yeMET, PhysParams P,
		int64_t tick, double tick_time, HeStiffItem *__restrict__ stiff, unsigned *__restrict__ nstiff,
		uint32_t *__restrict__ status) {
	const int a = tick_act[t] + blockIdx.x * blockDim.x + threadIdx.x;
	if (a >= tick_act[t + 1]) return;
	const uint32_t s0 = act_seg[a], s1 = act_seg[a + 1];
	double g0 = 0.0, g1 = 0.0, g2 = 0.0, heat = 0.0;
	int nh = 0;
	const double2 *acc2 = reinterpret_cast<const double2 *>(acc);
	for (uint32_t k = s0; k < s1; k++) {
		const double2 a = acc2[2 * (size_t)k];
		if (a.x >= 0.0) {
			const double2 b = acc2[2 * (size_t)k + 1];
			g0 += a.x;
			g1 += b.x;
			g2 += b.y;
			if (want_heat) heat += a.y;
			nh++;
		}
	}
	const uint32_t p = act_ipar[a];
	hits[p] += nh;
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
			return;
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

// The stiff helium particles of a tick, one thread each (their number is
// read on the device): the Rosenbrock finish from where the explicit steps
// stopped.
__global__ void __launch_bounds__(64) k_update_he_stiff(const HeStiffItem *__restrict__ stiff,
		const unsigned *__restrict__ nstiff, double *__restrict__ lambdaH, float *__restrict__ ie,
		int64_t *__restrict__ lasthit, PhysParams P, int64_t tick, uint32_t *__restrict__ status) {
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
		const float *__restrict__ yeMET, PhysParams P, int64_t tick, double tick_time, float *__restrict__ feat) {
	const int lo = tick_act[t];
	const int a = lo + blockIdx.x * blockDim.x + threadIdx.x;
	if (a >= tick_act[t + 1]) return;
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

__global__ void k_log_post(int t, const int32_t *__restrict__ tick_act, const uint32_t *__restrict__ act_ipar,
		const double *__restrict__ lambdaH, const float *__restrict__ ie, const float *__restrict__ yeMET,
		PhysParams P, const float *__restrict__ feat, float *__restrict__ out, size_t cap,
		unsigned long long *__restrict__ count) {
	const int lo = tick_act[t];
	const int a = lo + blockIdx.x * blockDim.x + threadIdx.x;
	if (a >= tick_act[t + 1]) return;
	const uint32_t p = act_ipar[a];
	const double lam1 = lambdaH[p];
	const double T1 = ieye2T(P, (double)ie[p], rn_dadd(rn_dsub(1.0, lam1), P.he_e));
	const float *f = feat + (size_t)(a - lo) * 8;
	const float y0 = (float)(surr_logit(lam1) - (double)f[2]);
	const float y1 = (float)(log10(fmax(T1, 1e-300)) - (double)f[1]);
	if (!isfinite(y0) || !isfinite(y1)) return;
	const unsigned long long row = atomicAdd(count, 1ull);
	if (row >= cap) return;
	float *o = out + row * 8;
	for (int i = 0; i < PSG_SURR_NFEAT; i++) o[i] = f[i];
	o[5] = y0;
	o[6] = y1;
	o[7] = 0.0f;
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

// The per-batch by-particle order: sort (tick, ipar) keys of all hits,
// give every hit its slot, list the distinct (tick, particle) pairs with the
// first slot of each, and the first pair of every tick. Layout of S_ACT:
// head, scan, act_ipar, act_seg (hb+1 each), tick_act (K+1, 16-aligned),
// act_key (hb+1, 16-aligned).
template <typename KT>
static int build_slots(psg_context *ctx, size_t nray, size_t R, size_t K, size_t nhit, int shift, int tbits,
		const int64_t *off64, const uint32_t *hit_ipar, int nacc, int *nact_out) {
	cudaStream_t st = ctx->stream;
	const size_t hb = nhit ? nhit : 1;
	KT *keys = (KT *)psg_scratch(ctx, S_KEYS, sizeof(KT) * 2 * hb);
	uint32_t *vals = (uint32_t *)psg_scratch(ctx, S_VALS, sizeof(uint32_t) * 2 * hb);
	uint32_t *slot = (uint32_t *)psg_scratch(ctx, S_SLOT, sizeof(uint32_t) * hb);
	double *acc = (double *)psg_scratch(ctx, S_ACC, sizeof(double) * hb * nacc);
	char *actm = (char *)psg_scratch(ctx, S_ACT, sizeof(int32_t) * 4 * (hb + 1) + sizeof(int32_t) * (K + 2)
			+ sizeof(KT) * (hb + 1) + 1024);
	if (!keys || !vals || !slot || !acc || !actm) return PSG_E_NOMEM;
	int32_t *head = (int32_t *)actm;
	int32_t *hscan = head + (hb + 1);
	uint32_t *act_ipar = (uint32_t *)(hscan + (hb + 1));
	uint32_t *act_seg = act_ipar + (hb + 1);
	int32_t *tick_act = (int32_t *)(((uintptr_t)(act_seg + hb + 1) + 15) & ~(uintptr_t)15);
	KT *act_key = (KT *)(((uintptr_t)(tick_act + K + 1) + 15) & ~(uintptr_t)15);
	int nact = 0;
	if (nhit) {
		k_slot_keys<KT><<<blocks(nray * 32, 256), 256, 0, st>>>(nray, (int)R, shift, off64, hit_ipar, keys, vals);
		PSG_CHECK_LAUNCH();
		const int endbit = shift + tbits;
		size_t tmp = 0;
		PSG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, keys, keys + hb, vals, vals + hb, (int64_t)nhit, 0, endbit, st));
		void *dt = psg_scratch(ctx, S_CUB, tmp);
		if (!dt) return PSG_E_NOMEM;
		PSG_CUDA(cub::DeviceRadixSort::SortPairs(dt, tmp, keys, keys + hb, vals, vals + hb, (int64_t)nhit, 0, endbit, st));
		k_slots<KT><<<blocks(nhit, 256), 256, 0, st>>>(nhit, keys + hb, vals + hb, slot, head);
		PSG_CHECK_LAUNCH();
		tmp = 0;
		PSG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, head, hscan, (int)nhit, st));
		dt = psg_scratch(ctx, S_CUB, tmp);
		if (!dt) return PSG_E_NOMEM;
		PSG_CUDA(cub::DeviceScan::ExclusiveSum(dt, tmp, head, hscan, (int)nhit, st));
		k_active<KT><<<blocks(nhit, 256), 256, 0, st>>>(nhit, shift, keys + hb, head, hscan, act_ipar, act_seg, act_key);
		PSG_CHECK_LAUNCH();
		ctx->launches += 3;
		int last_scan = 0, last_head = 0;
		PSG_CUDA(cudaMemcpyAsync(&last_scan, hscan + nhit - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
		PSG_CUDA(cudaMemcpyAsync(&last_head, head + nhit - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
		PSG_CUDA(cudaStreamSynchronize(st));
		nact = last_scan + last_head;
	}
	k_tick_bounds<KT><<<blocks(K + 1, 128), 128, 0, st>>>((int)K, shift, act_key, nact, act_seg, (uint32_t)nhit, tick_act);
	PSG_CHECK_LAUNCH();
	ctx->launches++;
	*nact_out = nact;
	return PSG_OK;
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
	const PhysParams P = psg_phys_params(ctx);
	const int want_heat = !ctx->flags.isothermal;
	// helium and/or secondary ionisation take the general deposit; helium
	// its own update
	const bool gen = !ctx->flags.h_only || ctx->flags.secondary_ionization;
	const bool helium = !ctx->flags.h_only;
	const int nacc = helium ? 4 : (want_heat ? 2 : 1);

	ctx->nkev = 0;
	ctx->launches = 0;
	PSG_CUDA(cudaEventRecord(ctx->ev[0], st));
	int rc = psg_trace_internal(ctx, d_rays, nray, 1);
	if (rc) return rc;
	int64_t *off64 = (int64_t *)ctx->scratch[S_OFFSETS].p;
	int64_t nhit64 = 0;
	PSG_CUDA(cudaMemcpyAsync(&nhit64, off64 + nray, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
	PSG_CUDA(cudaStreamSynchronize(st));
	const size_t nhit = (size_t)nhit64;
	const size_t hb = nhit ? nhit : 1;
	uint32_t *hit_ipar = (uint32_t *)ctx->scratch[S_HIT_IPAR].p;
	double *hit_kern = (double *)ctx->scratch[S_HIT_KERN].p;
	psg_mark_begin(ctx, PSG_K_SLOTS);
	// by-particle order of all hits
	int shift = 1;
	while (shift < 32 && (1ull << shift) < (unsigned long long)ctx->n) shift++;
	int tbits = 0;
	while ((1ull << tbits) < (unsigned long long)K) tbits++;
	int nact = 0;
	int rc2 = (shift + tbits <= 32) ? build_slots<uint32_t>(ctx, nray, R, K, nhit, shift, tbits, off64, hit_ipar,
			nacc, &nact)
		: build_slots<unsigned long long>(ctx, nray, R, K, nhit, shift, tbits, off64, hit_ipar, nacc, &nact);
	if (rc2) return rc2;
	double *acc = (double *)ctx->scratch[S_ACC].p;
	uint32_t *slot = (uint32_t *)ctx->scratch[S_SLOT].p;
	char *actm = (char *)ctx->scratch[S_ACT].p;
	int32_t *head = (int32_t *)actm;
	int32_t *hscan = head + (hb + 1);
	uint32_t *act_ipar = (uint32_t *)(hscan + (hb + 1));
	uint32_t *act_seg = act_ipar + (hb + 1);
	int32_t *tick_act = (int32_t *)(((uintptr_t)(act_seg + hb + 1) + 15) & ~(uintptr_t)15);
	(void)head;
	unsigned long long *d_nsat = ctx->d_counters + 1;
	double *d_lost = (double *)(ctx->d_counters + 2);
	PSG_CUDA(cudaMemsetAsync(d_nsat, 0, 16, st));
	psg_mark_end(ctx);
	PSG_CUDA(cudaEventRecord(ctx->ev[1], st));

	// the tick loop
	std::vector<int32_t> h_tick_act(K + 1);
	PSG_CUDA(cudaMemcpyAsync(h_tick_act.data(), tick_act, sizeof(int32_t) * (K + 1), cudaMemcpyDeviceToHost, st));
	// long / middle / short ray lists of the batch (ray order, so each tick's
	// rays are a run)
	unsigned long long *cls = (unsigned long long *)psg_scratch(ctx, S_COUNT, sizeof(unsigned long long) * 2 * (nray + 1));
	uint32_t *ray_lists = (uint32_t *)psg_scratch(ctx, S_RAYLIST, sizeof(uint32_t) * (nray + 1));
	if (!cls || !ray_lists) return PSG_E_NOMEM;
	unsigned long long *cls_scan = cls + (nray + 1);
	k_ray_class<<<blocks(nray, 256), 256, 0, st>>>(nray, off64, cls);
	PSG_CHECK_LAUNCH();
	{
		size_t tmp = 0;
		PSG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, cls, cls_scan, (int)nray, st));
		void *dt = psg_scratch(ctx, S_CUB, tmp);
		if (!dt) return PSG_E_NOMEM;
		PSG_CUDA(cub::DeviceScan::ExclusiveSum(dt, tmp, cls, cls_scan, (int)nray, st));
	}
	std::vector<unsigned long long> h_scan(nray), h_last(1);
	PSG_CUDA(cudaMemcpyAsync(h_scan.data(), cls_scan, sizeof(unsigned long long) * nray, cudaMemcpyDeviceToHost, st));
	PSG_CUDA(cudaMemcpyAsync(h_last.data(), cls + nray - 1, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
	PSG_CUDA(cudaStreamSynchronize(st));
	const unsigned long long tot = h_scan[nray - 1] + h_last[0];
	const int nlong_all = (int)(uint32_t)tot, nmid_all = (int)(uint32_t)(tot >> 32);
	uint32_t *long_rays = ray_lists, *mid_rays = ray_lists + nlong_all, *short_rays = mid_rays + nmid_all;
	k_ray_lists<<<blocks(nray, 256), 256, 0, st>>>(nray, cls, cls_scan, long_rays, mid_rays, short_rays);
	PSG_CHECK_LAUNCH();
	ctx->launches += 2;
	// per-particle sums, the long-segment lists and (not isothermal) the
	// integrator's work cursors and stiff lists
	int dev_sms = 148;
	cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, ctx->device);
	const bool iso = ctx->flags.isothermal != 0;
	const size_t na = (size_t)(h_tick_act[K] > 0 ? h_tick_act[K] : 1);
	size_t maxt = 1;
	for (size_t t = 0; t < K; t++) maxt = std::max<size_t>(maxt, (size_t)(h_tick_act[t + 1] - h_tick_act[t]));
	const bool euler = ctx->flags.euler != 0;
	// (the network does not model the recombination photons: on the spot only)
	const bool surr = !iso && !euler && ctx->surr_on && !ctx->flags.adiabatic && ctx->flags.on_the_spot &&
			ctx->flags.h_only;
	char *um = (char *)psg_scratch(ctx, S_UPD, sizeof(double) * 2 * na + sizeof(unsigned) * 3 * (K + 1)
			+ (iso ? 0 : sizeof(StiffItem) * maxt) + (surr ? sizeof(uint32_t) * maxt : 0) + 512);
	int32_t *aflag = (int32_t *)psg_scratch(ctx, S_ALONG, sizeof(int32_t) * (3 * (na + 1) + K + 1) + 512);
	if (!um || !aflag) return PSG_E_NOMEM;
	double *act_g = (double *)um;
	double *act_heat = act_g + na;
	unsigned *cursors = (unsigned *)(act_heat + na);
	unsigned *nstiff = cursors + (K + 1);
	unsigned *nrej = nstiff + (K + 1);
	StiffItem *stiff = (StiffItem *)(((uintptr_t)(nrej + K + 1) + 15) & ~(uintptr_t)15);
	uint32_t *rej = (uint32_t *)(stiff + (iso ? 0 : maxt));
	PSG_CUDA(cudaMemsetAsync(cursors, 0, sizeof(unsigned) * 3 * (K + 1), st));
	if (surr) PSG_CUDA(cudaMemsetAsync(ctx->d_counters + 8, 0, sizeof(unsigned long long), st));
	UpdRec *urec = nullptr;
	HeStiffItem *hstiff = nullptr;      // helium: the stiff particles of a tick
	if (helium) {
		hstiff = (HeStiffItem *)psg_scratch(ctx, S_REC, sizeof(HeStiffItem) * maxt);
		if (!hstiff) return PSG_E_NOMEM;
	} else if (!iso || euler) {
		urec = (UpdRec *)psg_scratch(ctx, S_REC, sizeof(UpdRec) * maxt);
		if (!urec) return PSG_E_NOMEM;
	}
	float *feat = nullptr;
	if (ctx->log_buf && !iso && !helium) {
		feat = (float *)psg_scratch(ctx, S_LOG, sizeof(float) * 8 * maxt);
		if (!feat) return PSG_E_NOMEM;
	}
	// the long segments of the batch, listed in order, and each tick's first
	int32_t *ascan = aflag + (na + 1);
	uint32_t *long_act = (uint32_t *)(ascan + (na + 1));
	int32_t *tick_long = (int32_t *)(long_act + (na + 1));
	k_act_class<<<blocks(na + 1, 256), 256, 0, st>>>(na, act_seg, aflag);
	PSG_CHECK_LAUNCH();
	{
		size_t tmp = 0;
		PSG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, aflag, ascan, (int)(na + 1), st));
		void *dt = psg_scratch(ctx, S_CUB, tmp);
		if (!dt) return PSG_E_NOMEM;
		PSG_CUDA(cub::DeviceScan::ExclusiveSum(dt, tmp, aflag, ascan, (int)(na + 1), st));
	}
	k_act_lists<<<blocks(na, 256), 256, 0, st>>>(na, aflag, ascan, long_act);
	PSG_CHECK_LAUNCH();
	k_tick_long<<<blocks(K + 1, 256), 256, 0, st>>>((int)K, tick_act, ascan, tick_long);
	PSG_CHECK_LAUNCH();
	ctx->launches += 4;
	std::vector<int32_t> h_tick_long(K + 1);
	PSG_CUDA(cudaMemcpyAsync(h_tick_long.data(), tick_long, sizeof(int32_t) * (K + 1), cudaMemcpyDeviceToHost, st));
	PSG_CUDA(cudaStreamSynchronize(st));
	// capped hits settled by the affine-map scan when the last batch had many
	const bool aff = ctx->sat_frac > 1e-3;
	for (size_t t = 0; t < K; t++) {
		const unsigned long long c0 = h_scan[t * R], c1 = (t + 1 < K) ? h_scan[(t + 1) * R] : tot;
		const int l0 = (int)(uint32_t)c0, m0 = (int)(uint32_t)(c0 >> 32);
		const int nlong = (int)(uint32_t)c1 - l0, nmid = (int)(uint32_t)(c1 >> 32) - m0;
		const int s0 = (int)(t * R) - l0 - m0;
		const int nshort = (int)R - nlong - nmid;
		const unsigned grid = (unsigned)(nlong + (nmid + 3) / 4 + (nshort + DEP_THREADS / 32 - 1) / (DEP_THREADS / 32));
		psg_mark_begin(ctx, PSG_K_DEPOSIT);
		if (grid && gen)
			k_deposit<true, false><<<grid, DEP_THREADS, 0, st>>>(d_rays, long_rays + l0, nlong, mid_rays + m0,
					nmid, short_rays + s0, nshort, off64, hit_ipar, hit_kern, slot, ctx->d_lambdaH, ctx->d_mass, P,
					want_heat, acc, nacc, d_nsat, d_lost);
		else if (grid && aff)
			k_deposit<false, true><<<grid, DEP_THREADS, 0, st>>>(d_rays, long_rays + l0, nlong, mid_rays + m0,
					nmid, short_rays + s0, nshort, off64, hit_ipar, hit_kern, slot, ctx->d_lambdaH, ctx->d_mass, P,
					want_heat, acc, nacc, d_nsat, d_lost);
		else if (grid)
			k_deposit<false, false><<<grid, DEP_THREADS, 0, st>>>(d_rays, long_rays + l0, nlong, mid_rays + m0,
					nmid, short_rays + s0, nshort, off64, hit_ipar, hit_kern, slot, ctx->d_lambdaH, ctx->d_mass, P,
					want_heat, acc, nacc, d_nsat, d_lost);
		PSG_CHECK_LAUNCH();
		psg_mark_end(ctx);
		const int nact_t = h_tick_act[t + 1] - h_tick_act[t];
		psg_mark_begin(ctx, PSG_K_UPDATE);
		if (nact_t > 0 && helium) {
			if (P.ygrec)
				k_update_he<true><<<blocks(nact_t, 128), 128, 0, st>>>((int)t, tick_act, act_ipar, act_seg, acc,
						want_heat, ctx->d_hits, ctx->d_lambdaH, ctx->d_ie, ctx->d_lasthit,
						ctx->d_rho, ctx->d_yeMET, P, first_tick + (int64_t)t, tick_time, hstiff, nstiff + t,
						ctx->d_status);
			else
				k_update_he<false><<<blocks(nact_t, 128), 128, 0, st>>>((int)t, tick_act, act_ipar, act_seg, acc,
						want_heat, ctx->d_hits, ctx->d_lambdaH, ctx->d_ie, ctx->d_lasthit,
						ctx->d_rho, ctx->d_yeMET, P, first_tick + (int64_t)t, tick_time, hstiff, nstiff + t,
						ctx->d_status);
			PSG_CHECK_LAUNCH();
			k_update_he_stiff<<<dev_sms, 64, 0, st>>>(hstiff, nstiff + t, ctx->d_lambdaH, ctx->d_ie, ctx->d_lasthit,
					P, first_tick + (int64_t)t, ctx->d_status);
			PSG_CHECK_LAUNCH();
			ctx->launches += 2;
		} else if (nact_t > 0) {
			const int64_t tick = first_tick + (int64_t)t;
			const int nl = h_tick_long[t + 1] - h_tick_long[t];
			const int lb = (nl + 7) / 8;
			const unsigned rgrid = (unsigned)(lb + (int)blocks(nact_t, 256));
			const double *gcarry = euler ? ctx->d_gcarry : nullptr;
			double *keep_g = (surr || feat) ? act_g : nullptr, *keep_heat = (surr || feat) ? act_heat : nullptr;
#define PSG_REDUCE(ISO_, REC_)                                                                              \
	k_reduce<ISO_, REC_><<<rgrid, 256, 0, st>>>((int)t, tick_act, act_ipar, act_seg, acc, want_heat, \
			long_act + h_tick_long[t], nl, lb, ctx->d_hits, keep_g, keep_heat, ctx->d_lambdaH, ctx->d_ie,      \
			ctx->d_lasthit, ctx->d_rho, ctx->d_yeMET, ctx->d_hstep, urec, gcarry, P, tick, tick_time,          \
			ctx->d_status)
			if (iso && !euler) {
				if (P.ygrec) PSG_REDUCE(true, true);
				else PSG_REDUCE(true, false);
			} else {
				if (P.ygrec) PSG_REDUCE(false, true);
				else PSG_REDUCE(false, false);
			}
#undef PSG_REDUCE
			PSG_CHECK_LAUNCH();
			ctx->launches++;
			if (euler) {
				k_update_euler<<<blocks(nact_t, 128), 128, 0, st>>>((int)t, tick_act, urec, ctx->d_lambdaH, ctx->d_ie,
						ctx->d_lasthit, ctx->d_gcarry, P, tick, ctx->d_status);
				PSG_CHECK_LAUNCH();
				ctx->launches++;
			} else if (!iso) {
				const unsigned qgrid = (unsigned)std::min<size_t>(blocks(nact_t, 256), (size_t)dev_sms * 8);
				if (feat) {
					k_log_pre<<<blocks(nact_t, 256), 256, 0, st>>>((int)t, tick_act, act_ipar, act_g, act_heat,
							ctx->d_lambdaH, ctx->d_ie, ctx->d_lasthit, ctx->d_rho, ctx->d_yeMET, P, tick, tick_time, feat);
					PSG_CHECK_LAUNCH();
				}
				if (surr) {
					// the network first; the integrator takes its rejects
					rc = psg_surrogate_tick(ctx, (int)t, nact_t, tick_act, act_ipar, act_g, act_heat, P, tick,
							tick_time, rej, nrej + t, dev_sms);
					if (rc) return rc;
					ctx->launches++;
				}
				if (P.ygrec) {
					k_update_queue<true><<<qgrid, 32 * UPD_WARPS, 0, st>>>((int)t, tick_act, urec, ctx->d_lambdaH,
							ctx->d_ie, ctx->d_lasthit, ctx->d_hstep, P, tick, cursors + t, stiff, nstiff + t, nullptr,
							nullptr, ctx->d_status);
					PSG_CHECK_LAUNCH();
					k_update_stiff<true><<<dev_sms, 64, 0, st>>>(stiff, nstiff + t, ctx->d_lambdaH, ctx->d_ie,
							ctx->d_lasthit, P, tick, ctx->d_status);
				} else {
					k_update_queue<false><<<qgrid, 32 * UPD_WARPS, 0, st>>>((int)t, tick_act, urec, ctx->d_lambdaH,
							ctx->d_ie, ctx->d_lasthit, ctx->d_hstep, P, tick, cursors + t, stiff, nstiff + t,
							surr ? rej : nullptr, surr ? nrej + t : nullptr, ctx->d_status);
					PSG_CHECK_LAUNCH();
					k_update_stiff<false><<<dev_sms, 64, 0, st>>>(stiff, nstiff + t, ctx->d_lambdaH, ctx->d_ie,
							ctx->d_lasthit, P, tick, ctx->d_status);
				}
				PSG_CHECK_LAUNCH();
				ctx->launches += 2;
				if (feat) {
					k_log_post<<<blocks(nact_t, 256), 256, 0, st>>>((int)t, tick_act, act_ipar, ctx->d_lambdaH,
							ctx->d_ie, ctx->d_yeMET, P, feat, ctx->log_buf, ctx->log_cap, ctx->log_count);
					PSG_CHECK_LAUNCH();
				}
			}
		}
		psg_mark_end(ctx);
		ctx->launches++;
	}
	PSG_CUDA(cudaEventRecord(ctx->ev[2], st));
	unsigned long long nsat = 0;
	PSG_CUDA(cudaMemcpyAsync(&nsat, d_nsat, sizeof(nsat), cudaMemcpyDeviceToHost, st));
	rc = check_status(ctx);      // (synchronises the stream)
	if (rc) return rc;
	ctx->sat_frac = nhit ? (double)nsat / (double)nhit : 0.0;
	if (stats) {
		double lost = 0;
		PSG_CUDA(cudaMemcpyAsync(&lost, d_lost, sizeof(lost), cudaMemcpyDeviceToHost, st));
		PSG_CUDA(cudaStreamSynchronize(st));
		float trace_ms = 0.f, tick_ms = 0.f;
		cudaEventElapsedTime(&trace_ms, ctx->ev[0], ctx->ev[1]);
		cudaEventElapsedTime(&tick_ms, ctx->ev[1], ctx->ev[2]);
		stats->hits = (double)nhit;
		stats->saturated = (double)nsat;
		stats->active = (double)nact;
		stats->lost_photons = lost;
		stats->trace_ms = trace_ms;
		stats->tick_ms = tick_ms;
		stats->launches = (double)ctx->launches;
		stats->surrogate_accepted = 0.0;
		stats->rec_rays = stats->rec_photons = 0.0;
		if (surr) {
			unsigned long long acc_n = 0;
			PSG_CUDA(cudaMemcpyAsync(&acc_n, ctx->d_counters + 8, sizeof(acc_n), cudaMemcpyDeviceToHost, st));
			PSG_CUDA(cudaStreamSynchronize(st));
			stats->surrogate_accepted = (double)acc_n;
		}
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
