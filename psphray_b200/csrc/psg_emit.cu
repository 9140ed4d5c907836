// Source rays on the device; replaces the source-ray half of emit_rays()
// loop.c:163-373 with psystem_weight_srcs() sources.c:67-78 and
// spec_gen_freq() spectra.c:50-60.
//
// Per tick the sources' weights (photons accumulated since each source last
// emitted) are summed in order into a CDF; every ray draws its source from
// it, each source's photons are split evenly over the rays that drew it
// (loop.c:305-320), and a source that drew a ray has emitted at this tick.
// These steps depend on the previous tick's draws, so one block walks the
// ticks of a batch in order (kernel k_emit_draw); the geometry and energy of
// every ray are then filled in parallel (k_emit_fill).
//
// Random numbers: Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel
// random numbers: as easy as 1, 2, 3", SC'11), counter = (ray index within
// the tick, tick low word, tick high word, stream), key = the 64-bit seed.
// A double uniform in [0,1) takes the top 53 bits of two 32-bit words. The
// reference draws from GSL's MT19937; this stream is the library's own and
// is restated in the oracle for the tests.
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "psg_internal.cuh"
#include "psg_philox.cuh"

namespace {

struct SrcDev {
	double pos[3], dir[3], a[3], b[3], radius;
	int type, specid, hist_off, hist_n;
};

// Offsets of the parts of ctx->d_emit.
struct EmitLayout {
	size_t src, hticks, hngd, lastemit, cursor, spec_off, spec_eng, spec_cdf, total;
};

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

EmitLayout emit_layout(int nsrc, int nhist, int nspec, int nspec_total) {
	EmitLayout L;
	size_t o = 0;
	L.src = o; o = align256(o + sizeof(SrcDev) * nsrc);
	L.hticks = o; o = align256(o + sizeof(int64_t) * nhist);
	L.hngd = o; o = align256(o + sizeof(double) * nhist);
	L.lastemit = o; o = align256(o + sizeof(int64_t) * nsrc);
	L.cursor = o; o = align256(o + sizeof(int32_t) * nsrc);
	L.spec_off = o; o = align256(o + sizeof(int32_t) * (nspec + 1));
	L.spec_eng = o; o = align256(o + sizeof(double) * nspec_total);
	L.spec_cdf = o; o = align256(o + sizeof(double) * nspec_total);
	L.total = o;
	return L;
}

struct EmitView {
	const SrcDev *src;
	const int64_t *hticks;
	const double *hngd;
	int64_t *lastemit;
	int32_t *cursor;
	const int32_t *spec_off;
	const double *spec_eng, *spec_cdf;
	int nsrc;
};

EmitView emit_view(const psg_context *ctx) {
	const EmitLayout L = emit_layout(ctx->nsrc, ctx->nhist_total, ctx->nspec, ctx->nspec_total);
	char *b = (char *)ctx->d_emit;
	EmitView v;
	v.src = (const SrcDev *)(b + L.src);
	v.hticks = (const int64_t *)(b + L.hticks);
	v.hngd = (const double *)(b + L.hngd);
	v.lastemit = (int64_t *)(b + L.lastemit);
	v.cursor = (int32_t *)(b + L.cursor);
	v.spec_off = (const int32_t *)(b + L.spec_off);
	v.spec_eng = (const double *)(b + L.spec_eng);
	v.spec_cdf = (const double *)(b + L.spec_cdf);
	v.nsrc = ctx->nsrc;
	return v;
}

// One block walks the K ticks in order: weights, their running sum, a source
// per ray, the per-source photon split, lastemit.
__global__ void __launch_bounds__(1024) k_emit_draw(EmitView E, size_t R, int K, int64_t first_tick,
		double tick_time, uint64_t seed, uint16_t *__restrict__ ray_src, double *__restrict__ tick_nph) {
	extern __shared__ double sm[];
	const int ns = E.nsrc;
	double *w = sm;
	double *cdf = sm + ns;
	unsigned *cnt = (unsigned *)(sm + 2 * ns);
	__shared__ int last_pos;
	for (int t = 0; t < K; t++) {
		const int64_t tick = first_tick + t;
		for (int i = threadIdx.x; i < ns; i += blockDim.x) {
			const SrcDev &S = E.src[i];
			int c = E.cursor[i];
			while (c < S.hist_n - 1 && E.hticks[S.hist_off + c + 1] <= tick) c++;   // advance_cursor()
			E.cursor[i] = c;
			w[i] = rn_dmul(rn_dmul(E.hngd[S.hist_off + c], (double)(tick - E.lastemit[i])), tick_time);
			cnt[i] = 0;
		}
		__syncthreads();
		if (threadIdx.x == 0) {
			double acc = 0.0;
			int lp = 0;
			for (int i = 0; i < ns; i++) {
				acc = rn_dadd(acc, w[i]);
				cdf[i] = acc;
				if (w[i] > 0.0) lp = i;
			}
			last_pos = lp;
		}
		__syncthreads();
		const double total = cdf[ns - 1];
		for (size_t r = threadIdx.x; r < R; r += blockDim.x) {
			uint32_t x[4];
			draw(x, (uint32_t)r, tick, 0u, seed);
			const double target = rn_dmul(u01(x[0], x[1]), total);
			int i = upper_index(cdf, 0, ns, target);
			if (i >= ns) i = last_pos;
			atomicAdd(&cnt[i], 1u);
			ray_src[(size_t)t * R + r] = (uint16_t)i;
		}
		__syncthreads();
		for (int i = threadIdx.x; i < ns; i += blockDim.x) {
			const unsigned c = cnt[i];
			tick_nph[(size_t)t * ns + i] = c ? rn_dmul(w[i], __ddiv_rn(1.0, (double)c)) : 0.0;
			if (c) E.lastemit[i] = tick;
		}
		__syncthreads();
	}
}

// Geometry and energy of every ray.
__global__ void k_emit_fill(EmitView E, size_t R, size_t K, int64_t first_tick, uint64_t seed, double length,
		const uint16_t *__restrict__ ray_src, const double *__restrict__ tick_nph, psg_ray *__restrict__ out) {
	const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
	if (idx >= R * K) return;
	const size_t t = idx / R, r = idx - t * R;
	const int64_t tick = first_tick + (int64_t)t;
	const int isrc = ray_src[idx];
	const SrcDev &S = E.src[isrc];
	psg_ray ray;
	ray.Nph = tick_nph[t * (size_t)E.nsrc + isrc];
	ray.length = length;
	if (S.type == PSG_SRC_POINT) {
		uint32_t x[4];
		draw(x, (uint32_t)r, tick, 1u, seed);
		const double c = rn_dsub(rn_dmul(2.0, u01(x[0], x[1])), 1.0);
		const double phi = rn_dmul(2.0 * 3.141592653589793, u01(x[2], x[3]));
		const double st = __dsqrt_rn(fmax(0.0, rn_dsub(1.0, rn_dmul(c, c))));
		double sp, cp;
		sincos(phi, &sp, &cp);
		ray.dir[0] = (float)rn_dmul(st, cp);
		ray.dir[1] = (float)rn_dmul(st, sp);
		ray.dir[2] = (float)c;
		for (int d = 0; d < 3; d++) ray.s[d] = (float)S.pos[d];
	} else {
		uint32_t x[4];
		draw(x, (uint32_t)r, tick, 3u, seed);
		const double u = rn_dsub(rn_dmul(2.0, u01(x[0], x[1])), 1.0);
		const double v = rn_dsub(rn_dmul(2.0, u01(x[2], x[3])), 1.0);
		for (int d = 0; d < 3; d++) {
			ray.dir[d] = (float)S.dir[d];
			ray.s[d] = (float)rn_dadd(rn_dadd(S.pos[d], rn_dmul(rn_dmul(u, S.a[d]), S.radius)),
					rn_dmul(rn_dmul(v, S.b[d]), S.radius));
		}
	}
	const int o0 = E.spec_off[S.specid], o1 = E.spec_off[S.specid + 1];
	if (o1 - o0 == 1) {
		ray.freq = E.spec_eng[o0];
	} else {
		uint32_t x[4];
		draw(x, (uint32_t)r, tick, 2u, seed);
		const double target = rn_dmul(u01(x[0], x[1]), E.spec_cdf[o1 - 1]);
		int i = upper_index(E.spec_cdf, o0, o1, target);
		if (i >= o1) i = o1 - 1;
		ray.freq = E.spec_eng[i];
	}
	out[idx] = ray;
}

// Emits R*K rays into the S_EMIT scratch; returns them in *d_out.
int emit_internal(psg_context *ctx, size_t R, size_t K, int64_t first_tick, double tick_time, psg_ray **d_out) {
	if (!ctx->d_emit || ctx->nsrc <= 0) return psg_fail(ctx, PSG_E_INVAL, "emit: no sources (psg_set_sources first)");
	if (ctx->n == 0) return psg_fail(ctx, PSG_E_INVAL, "emit: load particles first (the ray length is twice the box)");
	if (R == 0 || K == 0) return psg_fail(ctx, PSG_E_INVAL, "emit: empty batch");
	if (K >= (1u << 24) || R * K >= (size_t)INT32_MAX || R > UINT32_MAX)
		return psg_fail(ctx, PSG_E_OVERFLOW, "emit: batch too large");
	cudaStream_t st = ctx->stream;
	const size_t ray_bytes = align256(sizeof(psg_ray) * R * K);
	const size_t src_bytes = align256(sizeof(uint16_t) * R * K);
	const size_t nph_bytes = sizeof(double) * K * (size_t)ctx->nsrc;
	char *m = (char *)psg_scratch(ctx, S_EMIT, ray_bytes + src_bytes + nph_bytes);
	if (!m) return PSG_E_NOMEM;
	psg_ray *rays = (psg_ray *)m;
	uint16_t *ray_src = (uint16_t *)(m + ray_bytes);
	double *tick_nph = (double *)(m + ray_bytes + src_bytes);
	const EmitView E = emit_view(ctx);
	const size_t smem = (size_t)ctx->nsrc * (2 * sizeof(double) + sizeof(unsigned));
	if (smem > 48 * 1024)
		PSG_CUDA(cudaFuncSetAttribute(k_emit_draw, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
	k_emit_draw<<<1, 1024, smem, st>>>(E, R, (int)K, first_tick, tick_time, ctx->emit_seed, ray_src, tick_nph);
	PSG_CHECK_LAUNCH();
	const size_t n = R * K;
	k_emit_fill<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(E, R, K, first_tick, ctx->emit_seed,
			2.0 * ctx->boxsize, ray_src, tick_nph, rays);
	PSG_CHECK_LAUNCH();
	ctx->launches += 2;
	*d_out = rays;
	return PSG_OK;
}

}  // namespace

extern "C" int psg_set_sources(psg_context *ctx, const psg_source *srcs, int nsrc, const psg_spectrum *specs,
		int nspec, uint64_t seed) {
	if (!ctx) return PSG_E_INVAL;
	if (nsrc < 1 || nsrc > PSG_MAX_SOURCES || !srcs)
		return psg_fail(ctx, PSG_E_INVAL, "psg_set_sources: nsrc %d outside [1, %d]", nsrc, PSG_MAX_SOURCES);
	if (nspec < 1 || !specs) return psg_fail(ctx, PSG_E_INVAL, "psg_set_sources: no spectra");
	int nhist = 0, nspec_total = 0;
	for (int i = 0; i < nsrc; i++) {
		const psg_source &s = srcs[i];
		if (s.type != PSG_SRC_POINT && s.type != PSG_SRC_PLANE)
			return psg_fail(ctx, PSG_E_INVAL, "psg_set_sources: source %d has unknown type %d", i, s.type);
		if (s.specid < 0 || s.specid >= nspec)
			return psg_fail(ctx, PSG_E_INVAL, "psg_set_sources: source %d spectrum %d out of range", i, s.specid);
		if (s.nhist < 1 || !s.ticks || !s.ngamma_dot)
			return psg_fail(ctx, PSG_E_INVAL, "psg_set_sources: source %d has no luminosity history", i);
		for (int k = 0; k < s.nhist; k++)
			if (!(s.ngamma_dot[k] >= 0.0) || (k && s.ticks[k] < s.ticks[k - 1]))
				return psg_fail(ctx, PSG_E_INVAL, "psg_set_sources: source %d history entry %d invalid", i, k);
		nhist += s.nhist;
	}
	for (int j = 0; j < nspec; j++) {
		if (specs[j].n < 1 || !specs[j].eng || (specs[j].n > 1 && !specs[j].weight))
			return psg_fail(ctx, PSG_E_INVAL, "psg_set_sources: spectrum %d is empty", j);
		double tot = 0.0;
		for (int k = 0; k < specs[j].n && specs[j].n > 1; k++) {
			if (!(specs[j].weight[k] >= 0.0)) return psg_fail(ctx, PSG_E_INVAL, "psg_set_sources: spectrum %d weight %d < 0", j, k);
			tot += specs[j].weight[k];
		}
		if (specs[j].n > 1 && !(tot > 0.0)) return psg_fail(ctx, PSG_E_INVAL, "psg_set_sources: spectrum %d has zero weight", j);
		nspec_total += specs[j].n;
	}
	const EmitLayout L = emit_layout(nsrc, nhist, nspec, nspec_total);
	std::vector<char> h(L.total, 0);
	SrcDev *hs = (SrcDev *)(h.data() + L.src);
	int64_t *ht = (int64_t *)(h.data() + L.hticks);
	double *hn = (double *)(h.data() + L.hngd);
	int64_t *hl = (int64_t *)(h.data() + L.lastemit);
	int32_t *so = (int32_t *)(h.data() + L.spec_off);
	double *se = (double *)(h.data() + L.spec_eng);
	double *sc = (double *)(h.data() + L.spec_cdf);
	int ho = 0;
	for (int i = 0; i < nsrc; i++) {
		const psg_source &s = srcs[i];
		SrcDev d;
		memcpy(d.pos, s.pos, sizeof d.pos);
		memcpy(d.dir, s.dir, sizeof d.dir);
		memcpy(d.a, s.a, sizeof d.a);
		memcpy(d.b, s.b, sizeof d.b);
		d.radius = s.radius;
		d.type = s.type;
		d.specid = s.specid;
		d.hist_off = ho;
		d.hist_n = s.nhist;
		hs[i] = d;
		for (int k = 0; k < s.nhist; k++) {
			ht[ho + k] = s.ticks[k];
			hn[ho + k] = s.ngamma_dot[k];
		}
		ho += s.nhist;
		hl[i] = s.lastemit;
	}
	int o = 0;
	for (int j = 0; j < nspec; j++) {
		so[j] = o;
		double acc = 0.0;
		for (int k = 0; k < specs[j].n; k++) {
			se[o + k] = specs[j].eng[k];
			acc += specs[j].n > 1 ? specs[j].weight[k] : 1.0;
			sc[o + k] = acc;
		}
		o += specs[j].n;
	}
	so[nspec] = o;
	PSG_CUDA(cudaSetDevice(ctx->device));
	if (ctx->d_emit) {
		PSG_CUDA(cudaStreamSynchronize(ctx->stream));
		PSG_CUDA(cudaFree(ctx->d_emit));
		ctx->d_emit = nullptr;
	}
	ctx->nsrc = 0;
	PSG_CUDA(cudaMalloc(&ctx->d_emit, L.total));
	PSG_CUDA(cudaMemcpyAsync(ctx->d_emit, h.data(), L.total, cudaMemcpyHostToDevice, ctx->stream));
	PSG_CUDA(cudaStreamSynchronize(ctx->stream));
	ctx->nsrc = nsrc;
	ctx->nspec = nspec;
	ctx->nhist_total = nhist;
	ctx->nspec_total = nspec_total;
	ctx->emit_seed = seed;
	return PSG_OK;
}

extern "C" int psg_get_sources(psg_context *ctx, int64_t *lastemit, int32_t *cursor) {
	if (!ctx) return PSG_E_INVAL;
	if (!ctx->d_emit) return psg_fail(ctx, PSG_E_INVAL, "psg_get_sources: no sources");
	PSG_CUDA(cudaSetDevice(ctx->device));
	const EmitView E = emit_view(ctx);
	if (lastemit)
		PSG_CUDA(cudaMemcpyAsync(lastemit, E.lastemit, sizeof(int64_t) * ctx->nsrc, cudaMemcpyDeviceToHost, ctx->stream));
	if (cursor)
		PSG_CUDA(cudaMemcpyAsync(cursor, E.cursor, sizeof(int32_t) * ctx->nsrc, cudaMemcpyDeviceToHost, ctx->stream));
	PSG_CUDA(cudaStreamSynchronize(ctx->stream));
	return PSG_OK;
}

extern "C" int psg_emit_rays(psg_context *ctx, size_t R, size_t K, int64_t first_tick, double tick_time,
		psg_ray *rays) {
	if (!ctx) return PSG_E_INVAL;
	if (!rays) return psg_fail(ctx, PSG_E_INVAL, "psg_emit_rays: null output");
	PSG_CUDA(cudaSetDevice(ctx->device));
	psg_ray *d = nullptr;
	const int rc = emit_internal(ctx, R, K, first_tick, tick_time, &d);
	if (rc) return rc;
	PSG_CUDA(cudaMemcpyAsync(rays, d, sizeof(psg_ray) * R * K, cudaMemcpyDeviceToHost, ctx->stream));
	PSG_CUDA(cudaStreamSynchronize(ctx->stream));
	return PSG_OK;
}

extern "C" int psg_run_ticks_emit(psg_context *ctx, size_t R, size_t K, int64_t first_tick, double tick_time,
		psg_tick_stats *stats) {
	if (!ctx) return PSG_E_INVAL;
	if (!ctx->have_physics || !ctx->have_tree)
		return psg_fail(ctx, PSG_E_INVAL, "psg_run_ticks_emit: set physics, load particles and build the tree first");
	PSG_CUDA(cudaSetDevice(ctx->device));
	if (ctx->timing) PSG_CUDA(cudaEventRecord(ctx->ev[3], ctx->stream));
	psg_ray *d = nullptr;
	int rc = emit_internal(ctx, R, K, first_tick, tick_time, &d);
	if (rc) return rc;
	if (ctx->timing) PSG_CUDA(cudaEventRecord(ctx->ev[4], ctx->stream));
	rc = psg_run_ticks_device(ctx, d, R, K, first_tick, tick_time, stats);
	if (rc) return rc;
	if (stats) {
		stats->launches += 2;
		stats->kernel_launches[PSG_K_EMIT] = 2;
		float ms = 0.f;
		if (ctx->timing) cudaEventElapsedTime(&ms, ctx->ev[3], ctx->ev[4]);
		stats->kernel_ms[PSG_K_EMIT] = ms;
	}
	return PSG_OK;
}
