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

#include <vector>

#include "psg_internal.cuh"
#include "psg_solve.cuh"

namespace {

inline unsigned blocks(size_t n, int bs) { return (unsigned)((n + bs - 1) / bs); }

PhysParams phys_params(const psg_context *ctx) {
	PhysParams P{};
	P.ar = ctx->d_ar;
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
	return P;
}

// Column-density factor of each hit, kernel = sph_depth(b/h) / h^2
// (loop.c:429-445), computed once per batch; b is overwritten.
__global__ void k_hit_kernel(size_t nhit, const uint32_t *__restrict__ ipar, const float4 *__restrict__ psml,
		double *__restrict__ b_to_kern, PhysParams P) {
	const size_t h = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
	if (h >= nhit) return;
	const double sml = (double)psml[ipar[h]].w;
	const double sml_inv = __ddiv_rn(1.0, sml);
	const double r_h = rn_dmul(b_to_kern[h], sml_inv);
	b_to_kern[h] = rn_dmul(sph_depth(P, r_h), rn_dmul(sml_inv, sml_inv));
}

// (tick, ipar) keys for the by-particle order; one warp per ray.
__global__ void k_slot_keys(size_t nray, int nray_per_tick, const int64_t *__restrict__ off,
		const uint32_t *__restrict__ ipar, unsigned long long *__restrict__ keys,
		uint32_t *__restrict__ vals) {
	const size_t r = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) / 32;
	const int lane = threadIdx.x & 31;
	if (r >= nray) return;
	const unsigned long long t = (unsigned long long)(r / (size_t)nray_per_tick);
	for (int64_t h = off[r] + lane; h < off[r + 1]; h += 32) {
		keys[h] = (t << 32) | ipar[h];
		vals[h] = (uint32_t)h;
	}
}

__global__ void k_slots(size_t nhit, const unsigned long long *__restrict__ skeys,
		const uint32_t *__restrict__ svals, uint32_t *__restrict__ slot, int32_t *__restrict__ head) {
	const size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
	if (k >= nhit) return;
	slot[svals[k]] = (uint32_t)k;
	head[k] = (k == 0 || skeys[k] != skeys[k - 1]) ? 1 : 0;
}

__global__ void k_active(size_t nhit, const unsigned long long *__restrict__ skeys,
		const int32_t *__restrict__ head, const int32_t *__restrict__ scan,
		uint32_t *__restrict__ act_ipar, uint32_t *__restrict__ act_seg,
		unsigned long long *__restrict__ act_key) {
	const size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
	if (k >= nhit) return;
	if (!head[k]) return;
	const int a = scan[k];
	act_ipar[a] = (uint32_t)(skeys[k] & 0xFFFFFFFFull);
	act_seg[a] = (uint32_t)k;
	act_key[a] = skeys[k];
}

// first active entry of every tick (and the total at index nticks)
__global__ void k_tick_bounds(int nticks, const unsigned long long *__restrict__ act_key, int nact,
		uint32_t *__restrict__ act_seg, uint32_t nhit, int32_t *__restrict__ tick_act) {
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t > nticks) return;
	const unsigned long long want = (unsigned long long)t << 32;
	int lo = 0, hi = nact;
	while (lo < hi) {
		const int mid = (lo + hi) / 2;
		if (act_key[mid] < want) lo = mid + 1; else hi = mid;
	}
	tick_act[t] = lo;
	if (t == nticks) act_seg[nact] = nhit;
}

__device__ __forceinline__ double warp_incl_sum(double v, int lane) {
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		const double u = __shfl_up_sync(0xffffffffu, v, o);
		if (lane >= o) v += u;
	}
	return v;
}

__device__ __forceinline__ bool below_cutoff(double TM, double Nph) {
	return TM < 0.0 || __ddiv_rn(TM, Nph) < 1e-10;
}

// One block of DEP_THREADS per ray; hits are taken DEP_THREADS at a time.
// Within a chunk, optical depths are summed with a block-wide FP64 scan; the
// first hit whose absorption exceeds its neutral atoms (loop.c:482-485) or
// after which TM/Nph < 1e-10 (loop.c:585) is found with a block min, settled
// by its own thread, and the scan restarts after it.
#define DEP_THREADS 256
#define DEP_WARPS (DEP_THREADS / 32)

__global__ void __launch_bounds__(DEP_THREADS) k_deposit(const psg_ray *__restrict__ rays, size_t ray0, int nray,
		const int64_t *__restrict__ off, const uint32_t *__restrict__ hipar, const double *__restrict__ hkern,
		const uint32_t *__restrict__ slot, const double *__restrict__ lambdaH, const float *__restrict__ mass,
		PhysParams P, int want_heat, double *__restrict__ acc, double *__restrict__ acc_heat,
		unsigned long long *__restrict__ n_sat, double *__restrict__ lost) {
	__shared__ double s_wsum[DEP_WARPS];
	__shared__ int s_first;
	__shared__ double s_tm;
	const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
	const size_t r = ray0 + blockIdx.x;
	if (blockIdx.x >= (unsigned)nray) return;
	const int64_t h0 = off[r], h1 = off[r + 1];
	if (h1 == h0) return;
	const double Nph = rays[r].Nph;
	const double freq = rays[r].freq;
	const bool skip_ray = (Nph == 0.0);
	const double sigma = xs_get_HI(P, freq);
	const double heat_factor = rn_dmul(P.H_PER_MASS, fdim(freq, P.HI_ENERGY));
	double TM = Nph;
	bool done = skip_ray;
	unsigned nsat = 0;
	for (int64_t base = h0; base < h1; base += DEP_THREADS) {
		const int64_t h = base + tid;
		const bool valid = h < h1;
		double tau = 0.0, NHI = 0.0, NH_inv = 0.0, delta = -1.0;
		if (valid && !done) {
			const uint32_t p = hipar[h];
			const double NH = rn_dmul((double)mass[p], P.H_PER_MASS);
			NHI = rn_dmul(lambdaH[p], NH);
			tau = rn_dmul(sigma, rn_dmul(hkern[h], NHI));
			NH_inv = __ddiv_rn(1.0, NH);
		}
		int start = 0;
		while (!done && start < DEP_THREADS) {
			const bool part = valid && tid >= start && tau != 0.0;
			const double my_tau = part ? tau : 0.0;
			// block scan: warp scan, then the warp totals
			double wi = my_tau;
#pragma unroll
			for (int o = 1; o < 32; o <<= 1) {
				const double u = __shfl_up_sync(0xffffffffu, wi, o);
				if (lane >= o) wi += u;
			}
			double we = __shfl_up_sync(0xffffffffu, wi, 1);
			if (lane == 0) we = 0.0;
			if (lane == 31) s_wsum[wid] = wi;
			if (tid == 0) s_first = DEP_THREADS;
			__syncthreads();
			double woff = 0.0, total = 0.0;
			for (int k = 0; k < DEP_WARPS; k++) {
				const double v = s_wsum[k];
				if (k < wid) woff += v;
				total += v;
			}
			const double incl = woff + wi, excl = woff + we;
			const double TMj = TM * exp(-excl);
			double absorb = TMj * -expm1(-my_tau);
			const double TMafter = TM * exp(-incl);
			const bool capped = part && absorb > NHI;
			const bool cut = part && below_cutoff(TMafter, Nph);
			if (capped || cut) atomicMin(&s_first, tid);
			__syncthreads();
			const int f = s_first;
			if (part && tid < f) delta = rn_dmul(absorb, NH_inv);
			if (f == DEP_THREADS) {
				TM = TM * exp(-total);
				__syncthreads();     // s_wsum / s_first are rewritten by the next chunk
				break;
			}
			if (tid == f) {
				double TMnew = TMafter;
				if (capped) {
					absorb = NHI;
					TMnew = TMj - NHI;
					nsat++;
				}
				delta = rn_dmul(absorb, NH_inv);
				s_tm = TMnew;
			}
			__syncthreads();
			TM = s_tm;
			if (below_cutoff(TM, Nph)) done = true;
			start = f + 1;
			__syncthreads();
		}
		if (valid) {
			const uint32_t sl = slot[h];
			acc[sl] = delta;
			if (want_heat) acc_heat[sl] = delta >= 0.0 ? rn_dmul(heat_factor, delta) : 0.0;
		}
	}
	for (int o = 16; o > 0; o >>= 1) nsat += __shfl_down_sync(0xffffffffu, nsat, o);
	if (lane == 0 && nsat) atomicAdd(n_sat, (unsigned long long)nsat);
	if (tid == 0 && !skip_ray) atomicAdd(lost, TM);
}

// update_pars() loop.c:653-770 for the particles hit in tick t, one thread
// per particle. A particle's deposits are summed in slot order; segments
// longer than a warp (particles next to a source are hit by nearly every
// ray) are summed by the whole warp, lanes strided, then a fixed butterfly.
template <bool ISO>
__global__ void __launch_bounds__(256) k_update(int t, const int32_t *__restrict__ tick_act,
		const uint32_t *__restrict__ act_ipar, const uint32_t *__restrict__ act_seg,
		const double *__restrict__ acc, const double *__restrict__ acc_heat, int want_heat,
		double *__restrict__ lambdaH, float *__restrict__ ie, int32_t *__restrict__ hits,
		int64_t *__restrict__ lasthit, const float *__restrict__ rho, const float *__restrict__ yeMET,
		PhysParams P, int64_t tick, double tick_time, uint32_t *__restrict__ status) {
	const int lo = tick_act[t], hi = tick_act[t + 1];
	const int lane = threadIdx.x & 31;
	const int a = lo + blockIdx.x * blockDim.x + threadIdx.x;
	const bool mine = a < hi;
	if (__all_sync(0xffffffffu, !mine)) return;
	uint32_t p = 0, s0 = 0, s1 = 0;
	if (mine) {
		p = act_ipar[a];
		s0 = act_seg[a];
		s1 = act_seg[a + 1];
	}
	double g = 0.0, heat = 0.0;
	int nh = 0;
	const bool longseg = mine && (s1 - s0) > 32;
	if (mine && !longseg) {
		for (uint32_t k = s0; k < s1; k++) {
			const double d = acc[k];
			if (d >= 0.0) {
				g += d;
				if (want_heat) heat += acc_heat[k];
				nh++;
			}
		}
	}
	unsigned lm = __ballot_sync(0xffffffffu, longseg);
	while (lm) {
		const int l = __ffs(lm) - 1;
		lm &= lm - 1;
		const uint32_t b0 = __shfl_sync(0xffffffffu, s0, l), b1 = __shfl_sync(0xffffffffu, s1, l);
		double sg = 0.0, sh = 0.0;
		int sn = 0;
		for (uint32_t k = b0 + lane; k < b1; k += 32) {
			const double d = acc[k];
			if (d >= 0.0) {
				sg += d;
				if (want_heat) sh += acc_heat[k];
				sn++;
			}
		}
#pragma unroll
		for (int o = 16; o > 0; o >>= 1) {
			sg += __shfl_xor_sync(0xffffffffu, sg, o);
			sh += __shfl_xor_sync(0xffffffffu, sh, o);
			sn += __shfl_xor_sync(0xffffffffu, sn, o);
		}
		if (lane == l) { g = sg; heat = sh; nh = sn; }
	}
	if (!mine) return;
	const double time = rn_dmul((double)(tick - lasthit[p]), tick_time);
	const double lam0 = lambdaH[p];
	const double ie0 = (double)ie[p];
	const double T = ieye2T(P, ie0, rn_dadd(rn_dsub(1.0, lam0), P.he_e));
	const double nH = rn_dmul(P.H_PER_MASS, (double)rho[p]);
	double lam = lam0, e = ie0;
	uint32_t st;
	if (ISO) st = solve_step_iso(P, lam, (double)yeMET[p], g, time, nH, T);
	else st = solve_step(P, lam, e, (double)yeMET[p], g, heat, time, nH, T);
	lambdaH[p] = lam;
	if (ISO) {
		ie[p] = (float)Tye2ie(P, T, rn_dadd(rn_dsub(1.0, lam), P.he_e));
	} else if (!P.adiabatic) {
		ie[p] = (float)e;
	}
	lasthit[p] = tick;
	hits[p] += nh;
	if (st) atomicOr(status, st);
}

__global__ void k_step_evolve(psg_step *steps, size_t n, PhysParams P, uint32_t *status) {
	const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
	if (i >= n) return;
	psg_step s = steps[i];
	double lam = s.lambdaH, e = s.ie;
	const uint32_t st = solve_step(P, lam, e, s.yeMET, s.yGdepHI, s.heat, s.time, s.nH, s.T);
	s.lambdaH = lam;
	s.ie = e;
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

extern "C" int psg_run_ticks_device(psg_context *ctx, const psg_ray *d_rays, size_t R, size_t K,
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
	const PhysParams P = phys_params(ctx);
	const int want_heat = !ctx->flags.isothermal;

	ctx->nkev = 0;
	ctx->launches = 0;
	PSG_CUDA(cudaEventRecord(ctx->ev[0], st));
	int rc = psg_trace_internal(ctx, d_rays, nray, 0);
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
	if (nhit) {
		k_hit_kernel<<<blocks(nhit, 256), 256, 0, st>>>(nhit, hit_ipar, ctx->d_psml, hit_kern, P);
		PSG_CHECK_LAUNCH();
		ctx->launches++;
	}

	// by-particle order of all hits
	unsigned long long *keys = (unsigned long long *)psg_scratch(ctx, S_KEYS, sizeof(unsigned long long) * 2 * hb);
	uint32_t *vals = (uint32_t *)psg_scratch(ctx, S_VALS, sizeof(uint32_t) * 2 * hb);
	uint32_t *slot = (uint32_t *)psg_scratch(ctx, S_SLOT, sizeof(uint32_t) * hb);
	double *acc = (double *)psg_scratch(ctx, S_ACC, sizeof(double) * hb * (want_heat ? 2 : 1));
	char *actm = (char *)psg_scratch(ctx, S_ACT, (sizeof(int32_t) * 2 + sizeof(uint32_t) * 2 + 8) * (hb + 1)
			+ sizeof(int32_t) * (K + 2) + 1024);
	if (!keys || !vals || !slot || !acc || !actm) return PSG_E_NOMEM;
	double *acc_heat = want_heat ? acc + hb : nullptr;
	int32_t *head = (int32_t *)actm;
	int32_t *hscan = head + (hb + 1);
	uint32_t *act_ipar = (uint32_t *)(hscan + (hb + 1));
	uint32_t *act_seg = act_ipar + (hb + 1);
	unsigned long long *act_key = (unsigned long long *)(((uintptr_t)(act_seg + hb + 1) + 15) & ~(uintptr_t)15);
	int32_t *tick_act = (int32_t *)(act_key + hb + 1);
	int nact = 0;
	if (nhit) {
		k_slot_keys<<<blocks(nray * 32, 256), 256, 0, st>>>(nray, (int)R, off64, hit_ipar, keys, vals);
		PSG_CHECK_LAUNCH();
		int endbit = 32;
		while ((1ull << (endbit - 32)) < (unsigned long long)K) endbit++;
		size_t tmp = 0;
		PSG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, keys, keys + hb, vals, vals + hb, (int64_t)nhit, 0, endbit, st));
		void *dt = psg_scratch(ctx, S_CUB, tmp);
		if (!dt) return PSG_E_NOMEM;
		PSG_CUDA(cub::DeviceRadixSort::SortPairs(dt, tmp, keys, keys + hb, vals, vals + hb, (int64_t)nhit, 0, endbit, st));
		k_slots<<<blocks(nhit, 256), 256, 0, st>>>(nhit, keys + hb, vals + hb, slot, head);
		PSG_CHECK_LAUNCH();
		tmp = 0;
		PSG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, head, hscan, (int)nhit, st));
		dt = psg_scratch(ctx, S_CUB, tmp);
		if (!dt) return PSG_E_NOMEM;
		PSG_CUDA(cub::DeviceScan::ExclusiveSum(dt, tmp, head, hscan, (int)nhit, st));
		k_active<<<blocks(nhit, 256), 256, 0, st>>>(nhit, keys + hb, head, hscan, act_ipar, act_seg, act_key);
		PSG_CHECK_LAUNCH();
		ctx->launches += 3;
		int last_scan = 0, last_head = 0;
		PSG_CUDA(cudaMemcpyAsync(&last_scan, hscan + nhit - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
		PSG_CUDA(cudaMemcpyAsync(&last_head, head + nhit - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
		PSG_CUDA(cudaStreamSynchronize(st));
		nact = last_scan + last_head;
	}
	k_tick_bounds<<<blocks(K + 1, 128), 128, 0, st>>>((int)K, act_key, nact, act_seg, (uint32_t)nhit, tick_act);
	PSG_CHECK_LAUNCH();
	ctx->launches++;
	psg_mark_end(ctx);
	unsigned long long *d_nsat = ctx->d_counters + 1;
	double *d_lost = (double *)(ctx->d_counters + 2);
	PSG_CUDA(cudaMemsetAsync(d_nsat, 0, 16, st));
	PSG_CUDA(cudaEventRecord(ctx->ev[1], st));

	// the tick loop
	std::vector<int32_t> h_tick_act(K + 1);
	PSG_CUDA(cudaMemcpyAsync(h_tick_act.data(), tick_act, sizeof(int32_t) * (K + 1), cudaMemcpyDeviceToHost, st));
	PSG_CUDA(cudaStreamSynchronize(st));
	for (size_t t = 0; t < K; t++) {
		psg_mark_begin(ctx, PSG_K_DEPOSIT);
		k_deposit<<<(unsigned)R, DEP_THREADS, 0, st>>>(d_rays, t * R, (int)R, off64, hit_ipar, hit_kern,
				slot, ctx->d_lambdaH, ctx->d_mass, P, want_heat, acc, acc_heat, d_nsat, d_lost);
		PSG_CHECK_LAUNCH();
		psg_mark_end(ctx);
		const int nact_t = h_tick_act[t + 1] - h_tick_act[t];
		psg_mark_begin(ctx, PSG_K_UPDATE);
		if (nact_t > 0) {
			if (ctx->flags.isothermal)
				k_update<true><<<blocks(nact_t, 256), 256, 0, st>>>((int)t, tick_act, act_ipar, act_seg, acc,
						acc_heat, want_heat, ctx->d_lambdaH, ctx->d_ie, ctx->d_hits, ctx->d_lasthit, ctx->d_rho,
						ctx->d_yeMET, P, first_tick + (int64_t)t, tick_time, ctx->d_status);
			else
				k_update<false><<<blocks(nact_t, 256), 256, 0, st>>>((int)t, tick_act, act_ipar, act_seg, acc,
						acc_heat, want_heat, ctx->d_lambdaH, ctx->d_ie, ctx->d_hits, ctx->d_lasthit, ctx->d_rho,
						ctx->d_yeMET, P, first_tick + (int64_t)t, tick_time, ctx->d_status);
			PSG_CHECK_LAUNCH();
			ctx->launches++;
		}
		psg_mark_end(ctx);
		ctx->launches++;
	}
	PSG_CUDA(cudaEventRecord(ctx->ev[2], st));
	rc = check_status(ctx);
	if (rc) return rc;
	if (stats) {
		unsigned long long nsat = 0;
		double lost = 0;
		PSG_CUDA(cudaMemcpyAsync(&nsat, d_nsat, sizeof(nsat), cudaMemcpyDeviceToHost, st));
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
	k_step_evolve<<<blocks(n, 128), 128, 0, st>>>(d, n, phys_params(ctx), ctx->d_status);
	PSG_CHECK_LAUNCH();
	PSG_CUDA(cudaMemcpyAsync(steps, d, sizeof(psg_step) * n, cudaMemcpyDeviceToHost, st));
	PSG_CUDA(cudaStreamSynchronize(st));
	return check_status(ctx);
}
