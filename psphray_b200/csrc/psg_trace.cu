// Ray traversal; replaces rt_trace() raytrace.c:153-210 and the per-ray
// sort of trace() loop.c:375-386.
//
// The traversal walks the level-order copy of the octree (the 8 children of
// a cell contiguous), one warp per ray with a stack of crossed cells in
// shared memory; the set of crossed cells and the hits are the reference's
// parent/sibling walk's, found in another order. Hits go to per-ray slabs in
// discovery order and are then sorted per ray by (d, ipar).
#include <cub/cub.cuh>

#include <stdlib.h>
#include <string.h>

#include <vector>

#include "psg_internal.cuh"
#include "psg_bsort.cuh"
#include "psg_scan.cuh"
#include "psg_solve.cuh"

namespace {

// pluecker_() pluecker-sse.c:28-198. The reference's 8 hand-written sign
// classes reduce to one rule per axis and per axis pair (selected by the
// signs of dir); every product and difference rounds once, in float.
__device__ __forceinline__ bool segment_hits_box(const float dir[3], float dist, const float s2b[3],
		const float s2t[3]) {
	bool up[3];
#pragma unroll
	for (int a = 0; a < 3; a++) {
		up[a] = dir[a] > 0.0f;
		const float step = rn_fmul(dist, dir[a]);
		const float e2t = rn_fsub(s2t[a], step);
		const float e2b = rn_fsub(s2b[a], step);
		if (up[a] ? (s2t[a] < 0.0f) : (s2b[a] > 0.0f)) return false;
		if (up[a] ? (e2b > 0.0f) : (e2t < 0.0f)) return false;
	}
#pragma unroll
	for (int q = 0; q < 3; q++) {
		const int i = q == 2 ? 1 : 0;
		const int j = q == 0 ? 1 : 2;
		const float P = up[i] ? s2t[j] : s2b[j];
		const float R = up[i] ? s2b[j] : s2t[j];
		const float Q = up[j] ? s2b[i] : s2t[i];
		const float S = up[j] ? s2t[i] : s2b[i];
		if (rn_fmul(dir[i], P) < rn_fmul(dir[j], Q) || rn_fmul(dir[i], R) > rn_fmul(dir[j], S)) return false;
	}
	return true;
}

struct RayGeom {
	float s[3], dir[3], dist;
};

__device__ __forceinline__ RayGeom load_ray(const psg_ray *__restrict__ rays, size_t r) {
	RayGeom g;
	const psg_ray &ry = rays[r];
#pragma unroll
	for (int d = 0; d < 3; d++) { g.s[d] = ry.s[d]; g.dir[d] = ry.dir[d]; }
	g.dist = (float)ry.length;      // rt_trace() takes the length as float
	return g;
}

// The line test of raytrace.c:168-195: float differences and products,
// double sums (in the order the reference's build adds them: y and z
// first, then x); accepted iff sml^2 >= (dc - proj)(dc + proj).
// Candidates that miss by a wide margin are rejected in float first: the
// float estimate r2f = d2f - projf^2 carries at most ~12 roundings of
// relative size 2^-24 of d2 (about 7.2e-7 d2), so r2f - sml^2 > 1e-5 d2f
// guarantees the exact test rejects too; everything closer takes the exact
// double path, so the accepted set is the reference's.
__device__ __forceinline__ bool line_hits_particle(const RayGeom &g, float4 q, double &dc, double &r2) {
	const float dx = rn_fsub(q.x, g.s[0]), dy = rn_fsub(q.y, g.s[1]), dz = rn_fsub(q.z, g.s[2]);
	{
		const float pf = __fadd_rn(__fadd_rn(rn_fmul(dx, g.dir[0]), rn_fmul(dy, g.dir[1])), rn_fmul(dz, g.dir[2]));
		const float d2f = __fadd_rn(__fadd_rn(rn_fmul(dx, dx), rn_fmul(dy, dy)), rn_fmul(dz, dz));
		const float r2f = __fsub_rn(d2f, rn_fmul(pf, pf));
		if (__fsub_rn(r2f, rn_fmul(q.w, q.w)) > 1e-5f * d2f) return false;
	}
	// the three-term sums as the reference's build evaluates them: its
	// -ffast-math lets the compiler reassociate the loop into (y + z) + x,
	// which rounds differently from (x + y) + z in rare cases (1 ulp of d)
	const double proj = rn_dadd((double)rn_fmul(dx, g.dir[0]),
			rn_dadd((double)rn_fmul(dy, g.dir[1]), (double)rn_fmul(dz, g.dir[2])));
	const double d2 = rn_dadd((double)rn_fmul(dx, dx), rn_dadd((double)rn_fmul(dy, dy), (double)rn_fmul(dz, dz)));
	dc = __dsqrt_rn(d2);
	r2 = rn_dmul(rn_dsub(dc, proj), rn_dadd(dc, proj));
	return !((double)rn_fmul(q.w, q.w) < r2);
}

// Candidates listed in shared memory (leaf-order particle positions), tested
// 32 at a time; accepted hits go to the ray's slab in order of discovery.
__device__ __forceinline__ void test_candidates(const RayGeom &g, const int *list, int total,
		const float4 *__restrict__ lpsml, const uint32_t *__restrict__ lidx, size_t r, size_t scap,
		uint32_t *__restrict__ slab_ipar, double *__restrict__ slab_d, double *__restrict__ slab_b,
		uint32_t &nh, int lane, unsigned lt_mask) {
	for (int k0 = 0; k0 < total; k0 += 32) {
		const int k = k0 + lane;
		bool acc = false;
		double dc = 0.0, r2 = 0.0;
		uint32_t idx = 0;
		if (k < total) {
			const int p = list[k];
			idx = __ldg(&lidx[p]);
			if (!(idx & PSG_INVALID_BIT)) acc = line_hits_particle(g, __ldg(&lpsml[p]), dc, r2);
		}
		const unsigned bal = __ballot_sync(0xffffffffu, acc);
		if (acc) {
			const size_t q = nh + __popc(bal & lt_mask);
			if (q < scap) {
				const size_t o = r * scap + q;
				slab_ipar[o] = idx;
				slab_d[o] = dc;
				slab_b[o] = r2;      // (b = sqrt|r2| is taken in the sort, with every lane busy)
			}
		}
		nh += __popc(bal);
	}
}

// One warp per ray over the level-order tree, whose 8 children of a cell are
// contiguous. The warp keeps a stack (shared memory) of crossed internal
// cells; each step pops up to 4 of them and tests their 32 children at once,
// one per lane, with the reference's segment-box test; crossed internal
// children are pushed, crossed leaves list their particles for the line
// test. The cells tested are exactly the children of crossed cells, as in
// the reference's walk (raytrace.c:160-208); only the order differs, and the
// per-ray sort makes the output independent of it. The stack cannot exceed
// 4 + 28 entries per tree level; TR_STACK leaves room for 21 levels and an
// overflow would raise PSG_ST_STACK instead of losing cells.
#define TR_STACK 1024
#define TR_MAX_WARPS 16      // warps per block: ctx->tune.trace_warps, at most this

__global__ void __launch_bounds__(32 * TR_MAX_WARPS) k_trace_stack(const psg_ray *__restrict__ rays, size_t nray,
		const float4 *__restrict__ wlo, const float4 *__restrict__ whi,
		const float4 *__restrict__ lpsml, const uint32_t *__restrict__ lidx, int ppc,
		uint32_t *__restrict__ count, size_t scap, uint32_t *__restrict__ slab_ipar,
		double *__restrict__ slab_d, double *__restrict__ slab_b, unsigned long long *__restrict__ next_ray,
		uint32_t *__restrict__ status, const unsigned *__restrict__ nlim) {
	extern __shared__ int tr_smem[];
	// rays past *nlim (when given: the recombination path's emitted count)
	// are not traced; their counts stay as zeroed
	if (nlim) nray = min(nray, (size_t)*nlim);
	const int lane = threadIdx.x & 31;
	const int wib = threadIdx.x >> 5;
	int *stack = tr_smem + wib * (TR_STACK + 32 * ppc + 32);
	int *list = stack + TR_STACK;      // candidates waiting for a full round of 32
	// persistent warps: each takes the next ray from a shared counter, so a
	// block never idles behind its longest ray
	for (;;) {
	unsigned long long rr = 0;
	if (lane == 0) rr = atomicAdd(next_ray, 1ull);
	rr = __shfl_sync(0xffffffffu, rr, 0);
	if (rr >= nray) break;
	const size_t r = (size_t)rr;
	const RayGeom g = load_ray(rays, r);
	const unsigned lt_mask = (1u << lane) - 1u;
	uint32_t nh = 0;
	int sp = 0, nbuf = 0;
	bool overflow = false;
	{
		const float4 lo = __ldg(&wlo[0]), hi = __ldg(&whi[0]);
		const float s2b[3] = {rn_fsub(lo.x, g.s[0]), rn_fsub(lo.y, g.s[1]), rn_fsub(lo.z, g.s[2])};
		const float s2t[3] = {rn_fsub(hi.x, g.s[0]), rn_fsub(hi.y, g.s[1]), rn_fsub(hi.z, g.s[2])};
		if (segment_hits_box(g.dir, g.dist, s2b, s2t)) {
			const int w = __float_as_int(lo.w);
			if (w >= 0) {
				if (lane == 0) stack[0] = w;
				sp = 1;
			} else {
				const int cnt = min(-1 - w, ppc), ps = __float_as_int(hi.w);
				for (int k = lane; k < cnt; k += 32) list[k] = ps + k;
				__syncwarp();
				test_candidates(g, list, cnt, lpsml, lidx, r, scap, slab_ipar, slab_d, slab_b, nh, lane, lt_mask);
			}
		}
	}
	__syncwarp();
	while (sp > 0) {
		const int k = min(sp, 4);
		const int node = lane >> 3;
		const bool valid = node < k;
		const int c = valid ? stack[sp - k + node] + (lane & 7) : 0;
		__syncwarp();
		sp -= k;
		float4 lo = make_float4(0.f, 0.f, 0.f, 0.f), hi = lo;
		bool hit = false;
		if (valid) {
			lo = __ldg(&wlo[c]);
			hi = __ldg(&whi[c]);
			const float s2b[3] = {rn_fsub(lo.x, g.s[0]), rn_fsub(lo.y, g.s[1]), rn_fsub(lo.z, g.s[2])};
			const float s2t[3] = {rn_fsub(hi.x, g.s[0]), rn_fsub(hi.y, g.s[1]), rn_fsub(hi.z, g.s[2])};
			hit = segment_hits_box(g.dir, g.dist, s2b, s2t);
		}
		const int w = __float_as_int(lo.w);
		const bool internal = hit && w >= 0;
		const unsigned bi = __ballot_sync(0xffffffffu, internal);
		if (internal) {
			const int pos = sp + __popc(bi & lt_mask);
			if (pos < TR_STACK) stack[pos] = w;
		}
		sp += __popc(bi);
		if (sp > TR_STACK) { overflow = true; sp = TR_STACK; }
		const int cnt = (hit && w < 0) ? min(-1 - w, ppc) : 0;
		int cs = cnt;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			const int t = __shfl_up_sync(0xffffffffu, cs, o);
			if (lane >= o) cs += t;
		}
		const int total = __shfl_sync(0xffffffffu, cs, 31);
		if (cnt) {
			const int ps = __float_as_int(hi.w), base = nbuf + cs - cnt;
			for (int q = 0; q < cnt; q++) list[base + q] = ps + q;
		}
		nbuf += total;
		__syncwarp();
		// line tests only in full rounds of 32; the rest waits in the list
		if (nbuf >= 32) {
			const int full = nbuf & ~31, rem = nbuf - full;
			test_candidates(g, list, full, lpsml, lidx, r, scap, slab_ipar, slab_d, slab_b, nh, lane, lt_mask);
			__syncwarp();
			const int keep = lane < rem ? list[full + lane] : 0;
			__syncwarp();
			if (lane < rem) list[lane] = keep;
			nbuf = rem;
			__syncwarp();
		}
	}
	if (nbuf) test_candidates(g, list, nbuf, lpsml, lidx, r, scap, slab_ipar, slab_d, slab_b, nh, lane, lt_mask);
	if (lane == 0) {
		count[r] = nh;
		if (overflow) atomicOr(status, PSG_ST_STACK);
	}
	__syncwarp();
	}
}

// With cap (a call without host reads), a total above the hit buffers'
// capacity empties every list instead (nothing downstream reads past cap)
// and flags the status word for the host to redo the call; the call's
// largest total is kept in *tickmax.
__global__ void k_offsets64(const unsigned long long *__restrict__ scan, const uint32_t *__restrict__ count,
		size_t nray, int64_t *__restrict__ off64,
		unsigned long long *__restrict__ maxcount, size_t cap, unsigned long long *__restrict__ tickmax,
		uint32_t *__restrict__ status) {
	const size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
	if (r > nray) return;
	// scan holds the exclusive scan over nray+1 entries (count[nray] = 0)
	const bool over = cap && (size_t)scan[nray] > cap;
	off64[r] = over ? 0 : scan[r];
	if (r < nray) {
		atomicMax(maxcount, (unsigned long long)count[r]);
	} else {
		maxcount[1] = scan[r];       // the hit total, read with the longest list
		if (cap) {
			atomicMax(tickmax, (unsigned long long)scan[r]);
			if (over) atomicOr(status, PSG_ST_SLAB);
		}
	}
}

// The caller's index of internal particle i (order: null when the arrays
// are still in caller order); ties in d are broken by it.
__device__ __forceinline__ uint32_t caller_index(const uint32_t *__restrict__ order, uint32_t i) {
	return order ? order[i] : i;
}

// The hit at slab position p of a ray as the sorted list's entry h (the slab
// holds b^2; b = sqrt|b^2| here); with want_kern b becomes the
// column-density factor sph_depth(b/h)/h^2 (loop.c:429-445).
__device__ __forceinline__ void put_sorted_hit(int64_t h, uint32_t p, const uint32_t *__restrict__ raw_ipar,
		const double *__restrict__ raw_d, const double *__restrict__ raw_b, uint32_t *__restrict__ out_ipar,
		double *__restrict__ out_d, double *__restrict__ out_b, int want_kern, const float4 *__restrict__ psml,
		const PhysParams &P) {
	const uint32_t ip = raw_ipar[p];
	const double b = __dsqrt_rn(fabs(raw_b[p]));      // the slab holds the squared distance
	out_ipar[h] = ip;
	out_d[h] = raw_d[p];
	if (want_kern) {
		const double sml = (double)psml[ip].w;
		const double inv = __ddiv_rn(1.0, sml);
		out_b[h] = rn_dmul(sph_depth(P, rn_dmul(b, inv)), rn_dmul(inv, inv));
	} else {
		out_b[h] = b;
	}
}

// Per-ray sort by (d, ipar), one ray per block of TPR threads holding IPT
// hits each: a block radix sort (passes of 4 bits) on d mapped to KEY_BITS
// bits over the ray's own range of d (a monotone map) -- 12 bits for up to
// 1024 hits, 16 up to 4096, 20 beyond, so that about n^2 / 2^(bits+1) pairs
// share a key -- and the few runs of equal keys are then insertion-sorted
// on the exact (d, ipar) -- the reference's d
// order (loop.c:783-787) with ties broken by the caller's particle index. With want_kern the b column is replaced by the
// column-density factor sph_depth(b/h)/h^2 of loop.c:429-445.
template <int TPR, int IPT>
__global__ void __launch_bounds__(TPR) k_sort_block(const uint32_t *__restrict__ list,
		const unsigned long long *__restrict__ d_nlist,
		const int64_t *__restrict__ off, size_t scap, const uint32_t *__restrict__ slab_ipar,
		const double *__restrict__ slab_d, const double *__restrict__ slab_b, uint32_t *__restrict__ out_ipar,
		double *__restrict__ out_d, double *__restrict__ out_b, int want_kern, const float4 *__restrict__ psml,
		PhysParams P, const uint32_t *__restrict__ order, size_t slab_r0) {
	constexpr int NMAX = TPR * IPT;
	using Sort = cub::BlockRadixSort<uint32_t, TPR, IPT, uint32_t, 4>;
	struct Smem {
		typename Sort::TempStorage sort;
		uint32_t key[NMAX];
		uint32_t pos[NMAX];
		double lo[TPR / 32], hi[TPR / 32];
	};
	extern __shared__ __align__(16) char sort_smem[];
	Smem &sm = *reinterpret_cast<Smem *>(sort_smem);
	// a persistent grid: the class's ray count is read here, so the launch
	// needs no count from the host
	const unsigned long long nlist = *d_nlist;
	for (unsigned long long li = blockIdx.x; li < nlist; li += gridDim.x) {
	const size_t r = list[li];
	const int64_t h0 = off[r];
	const int n = (int)(off[r + 1] - h0);
	const uint32_t *raw_ipar = slab_ipar + (r - slab_r0) * scap;
	const double *raw_d = slab_d + (r - slab_r0) * scap, *raw_b = slab_b + (r - slab_r0) * scap;
	// keys: d mapped onto 24 bits over the ray's [min, max] (monotone, so
	// equal keys only ever hide an order the fix-up below restores)
	double dv[IPT];
	double dlo = 1e300, dhi = -1e300;
#pragma unroll
	for (int u = 0; u < IPT; u++) {
		const int i = threadIdx.x * IPT + u;
		dv[u] = i < n ? raw_d[i] : 0.0;
		if (i < n) {
			dlo = fmin(dlo, dv[u]);
			dhi = fmax(dhi, dv[u]);
		}
	}
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) {
		dlo = fmin(dlo, __shfl_xor_sync(0xffffffffu, dlo, o));
		dhi = fmax(dhi, __shfl_xor_sync(0xffffffffu, dhi, o));
	}
	if ((threadIdx.x & 31) == 0) {
		sm.lo[threadIdx.x >> 5] = dlo;
		sm.hi[threadIdx.x >> 5] = dhi;
	}
	__syncthreads();
#pragma unroll
	for (int w = 0; w < TPR / 32; w++) {
		dlo = fmin(dlo, sm.lo[w]);
		dhi = fmax(dhi, sm.hi[w]);
	}
	constexpr int KEY_BITS = NMAX <= 1024 ? 12 : (NMAX <= 4096 ? 16 : 20);
	constexpr uint32_t KEY_MAX = (1u << KEY_BITS) - 1u;
	const double scale = dhi > dlo ? (double)KEY_MAX / (dhi - dlo) : 0.0;
	uint32_t k[IPT], v[IPT];
#pragma unroll
	for (int u = 0; u < IPT; u++) {
		const int i = threadIdx.x * IPT + u;
		// padding takes the largest key; the sort is stable and padding
		// follows every real item, so it stays behind them
		k[u] = i < n ? min((uint32_t)((dv[u] - dlo) * scale), KEY_MAX) : KEY_MAX;
		v[u] = (uint32_t)i;
	}
	Sort(sm.sort).Sort(k, v, 0, KEY_BITS);
	__syncthreads();
#pragma unroll
	for (int u = 0; u < IPT; u++) {
		const int i = threadIdx.x * IPT + u;
		sm.key[i] = k[u];
		sm.pos[i] = v[u];
	}
	__syncthreads();
	// exact order inside runs of equal float keys
	for (int i = threadIdx.x; i + 1 < n; i += TPR) {
		if (sm.key[i] != sm.key[i + 1] || (i > 0 && sm.key[i - 1] == sm.key[i])) continue;
		int e = i + 1;
		while (e + 1 < n && sm.key[e + 1] == sm.key[i]) e++;
		for (int a = i + 1; a <= e; a++) {
			const uint32_t pa = sm.pos[a];
			const double da = raw_d[pa];
			const uint32_t ia = caller_index(order, raw_ipar[pa]);
			int c = a;
			while (c > i) {
				const uint32_t pc = sm.pos[c - 1];
				const double dc = raw_d[pc];
				if (dc < da || (dc == da && caller_index(order, raw_ipar[pc]) < ia)) break;
				sm.pos[c] = pc;
				c--;
			}
			sm.pos[c] = pa;
		}
	}
	__syncthreads();
	for (int i = threadIdx.x; i < n; i += TPR)
		put_sorted_hit(h0 + i, sm.pos[i], raw_ipar, raw_d, raw_b, out_ipar, out_d, out_b, want_kern, psml, P);
	__syncthreads();     // shared memory is reused by the next ray
	}
}

template <int TPR, int IPT>
size_t sort_smem_bytes() {
	return sizeof(typename cub::BlockRadixSort<uint32_t, TPR, IPT, uint32_t, 4>::TempStorage) + 8 * TPR * IPT +
			16 * (TPR / 32) + 128;
}

// Rays with more hits than the largest class (PSG_SORT_MAX), a block of
// LONG_NT threads each, persistent over their list: the hits as (d, caller
// index << 32 | slab position) pairs in tmp (the two halves, at the ray's
// list offset), sorted by block_sort_global on exactly the order of the
// class sorts -- d, then the caller's index.
#define LONG_NT 1024
struct LongHit {
	double d;
	unsigned long long ck;
};
struct LongHitLess {
	__device__ __forceinline__ bool operator()(const LongHit &x, const LongHit &y) const {
		return x.d < y.d || (x.d == y.d && x.ck < y.ck);
	}
};
__global__ void __launch_bounds__(LONG_NT) k_sort_long(const uint32_t *__restrict__ list,
		const unsigned long long *__restrict__ d_nlist, const int64_t *__restrict__ off, size_t scap,
		const uint32_t *__restrict__ slab_ipar, const double *__restrict__ slab_d, const double *__restrict__ slab_b,
		uint32_t *__restrict__ out_ipar, double *__restrict__ out_d, double *__restrict__ out_b, int want_kern,
		const float4 *__restrict__ psml, PhysParams P, const uint32_t *__restrict__ order, LongHit *tmp, size_t hb,
		size_t slab_r0) {
	__shared__ LongHit tile[2 * LONG_NT];
	const LongHit pad{__longlong_as_double(0x7ff0000000000000ll), ~0ull};
	const unsigned long long nlist = *d_nlist;
	for (unsigned long long li = blockIdx.x; li < nlist; li += gridDim.x) {
		const size_t r = list[li];
		const int64_t h0 = off[r];
		const int64_t n = off[r + 1] - h0;
		const uint32_t *raw_ipar = slab_ipar + (r - slab_r0) * scap;
		const double *raw_d = slab_d + (r - slab_r0) * scap, *raw_b = slab_b + (r - slab_r0) * scap;
		LongHit *a = tmp + h0;
		for (int64_t i = threadIdx.x; i < n; i += LONG_NT)
			a[i] = LongHit{raw_d[i], (unsigned long long)caller_index(order, raw_ipar[i]) << 32 | (unsigned long long)i};
		const LongHit *f = block_sort_global<LONG_NT>(a, tmp + hb + h0, n, tile, pad, LongHitLess());
		for (int64_t i = threadIdx.x; i < n; i += LONG_NT)
			put_sorted_hit(h0 + i, (uint32_t)f[i].ck, raw_ipar, raw_d, raw_b, out_ipar, out_d, out_b, want_kern,
					psml, P);
		__syncthreads();
	}
}

// Size classes of the ray sort: class c holds rays with at most
// kSortClassMax[c] hits (and more than the previous class's bound).
// size classes of the per-ray sort (threads x items per thread):
// 32x2, 32x4, 64x4, 128x4, 128x8, 256x8, 256x16, 512x16
#define SORT_NCLS 8
__constant__ int kSortBounds[SORT_NCLS] = {64, 128, 256, 512, 1024, 2048, 4096, PSG_SORT_MAX};

// rays [r0, nray) into the size classes' lists
__global__ void k_sort_classify(size_t r0, size_t nray, const int64_t *__restrict__ off, uint32_t *__restrict__ lists,
		size_t stride, unsigned long long *__restrict__ nclass, unsigned long long *__restrict__ nlong) {
	const size_t r = r0 + blockIdx.x * (size_t)blockDim.x + threadIdx.x;
	if (r >= nray) return;
	const int64_t n = off[r + 1] - off[r];
	if (n == 0) return;
	if (n > PSG_SORT_MAX) {      // the long list, after the classes'
		const unsigned long long k = atomicAdd(nlong, 1ull);
		lists[SORT_NCLS * stride + k] = (uint32_t)r;
		return;
	}
	int c = 0;
	while (c < SORT_NCLS - 1 && n > kSortBounds[c]) c++;
	const unsigned long long k = atomicAdd(&nclass[c], 1ull);
	lists[c * stride + k] = (uint32_t)r;
}

inline unsigned blocks(size_t n, int bs) { return (unsigned)((n + bs - 1) / bs); }

// S_COUNT during a traversal: the hit counts (nray + 1, u32), then their
// exclusive scan (nray + 2, u64) at the next 16-byte boundary
size_t count_bytes(size_t nray) { return 16 * ((sizeof(uint32_t) * (nray + 1) + 15) / 16) + 8 * (nray + 2) + 64; }
unsigned long long *count_scan(uint32_t *count, size_t nray) {
	return (unsigned long long *)((char *)count + 16 * ((sizeof(uint32_t) * (nray + 1) + 15) / 16));
}

}  // namespace

// Hit counts clamped to the slab capacity for the offsets (the slabs hold
// no more); the longest list of the call kept in *callmax, and a clamped list
// flagged in the status word (PSG_ST_SLAB) so the host redoes the call
// with larger slabs.
__global__ void k_count_clamp(size_t nray, size_t scap, uint32_t *__restrict__ count,
		unsigned long long *__restrict__ callmax, uint32_t *__restrict__ status) {
	const size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
	if (r >= nray) return;
	const uint32_t c = count[r];
	if (c > scap) {
		count[r] = (uint32_t)scap;
		atomicOr(status, PSG_ST_SLAB);
	}
	if (c) atomicMax(callmax, (unsigned long long)c);
}

namespace {
// The counts of a recombination tick after its traversal: the source rays'
// from the call's traced source rays (the tick is B->k of the call), the
// emitted rays' clamped to the slabs (as k_count_clamp).
__global__ void k_rec_counts(const PsgBatchDev *__restrict__ B, size_t R, const int64_t *__restrict__ src_off,
		size_t cap_rec, size_t scap, uint32_t *__restrict__ count, unsigned long long *__restrict__ callmax,
		uint32_t *__restrict__ status) {
	const int64_t base = B->k * (int64_t)R;
	for (size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x; r < R + cap_rec;
			r += (size_t)gridDim.x * blockDim.x) {
		if (r < R) {
			count[r] = (uint32_t)(src_off[base + (int64_t)r + 1] - src_off[base + (int64_t)r]);
			continue;
		}
		const uint32_t c = count[r];
		if (c > scap) {
			count[r] = (uint32_t)scap;
			atomicOr(status, PSG_ST_SLAB);
		}
		if (c) atomicMax(callmax, (unsigned long long)c);
	}
}
// their sorted hits into the tick's lists, a warp per ray (nothing when the
// tick's offsets were emptied for exceeding the capacity)
__global__ void k_copy_src_hits(const PsgBatchDev *__restrict__ B, size_t R, const int64_t *__restrict__ src_off,
		const uint32_t *__restrict__ src_ipar, const double *__restrict__ src_kern, const int64_t *__restrict__ off,
		uint32_t *__restrict__ hit_ipar, double *__restrict__ hit_kern) {
	const size_t r = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) / 32;
	const int lane = threadIdx.x & 31;
	if (r >= R) return;
	const int64_t base = B->k * (int64_t)R + (int64_t)r;
	const int64_t s0 = src_off[base];
	const int64_t n = min(src_off[base + 1] - s0, off[r + 1] - off[r]);
	const int64_t d0 = off[r];
	for (int64_t i = lane; i < n; i += 32) {
		hit_ipar[d0 + i] = src_ipar[s0 + i];
		hit_kern[d0 + i] = src_kern[s0 + i];
	}
}
}  // namespace

struct SrcHits {
	const int64_t *off;
	const uint32_t *ipar;
	const double *kern;
};
static SrcHits src_hits(psg_context *ctx) {
	char *m = (char *)ctx->scratch[S_SRCHIT].p;
	SrcHits h;
	h.off = (const int64_t *)m;
	h.kern = (const double *)(m + sizeof(int64_t) * (ctx->src_nray + 1));
	h.ipar = (const uint32_t *)(h.kern + ctx->src_nhit);
	return h;
}

// All source rays of a recombination call traced and sorted (with the
// column-density factor) before its ticks run; kept in S_SRCHIT. One host
// synchronisation (the traversal's).
int psg_trace_src_batch(psg_context *ctx, const psg_ray *d_rays, size_t nray) {
	PsgTraceFill tf;
	int rc = psg_trace_fill(ctx, d_rays, nray, &tf);
	if (!rc) rc = psg_trace_sort_prepare(ctx, nray, tf.nhit, tf.maxcount);
	if (!rc) rc = psg_trace_sort_enqueue(ctx, nray, tf.nhit, tf.maxcount, 1, 0);
	if (rc) return rc;
	// the layout depends on a grow-only capacity, not on this call's hit
	// total, so that calls of similar totals share one captured tick graph
	if (tf.nhit > ctx->src_nhit || nray != ctx->src_nray) {
		size_t c = std::max(tf.nhit + tf.nhit / 8, ctx->src_nhit);
		c = (c + 65535) & ~(size_t)65535;
		ctx->src_nhit = c;
	}
	char *m = (char *)psg_scratch(ctx, S_SRCHIT, sizeof(int64_t) * (nray + 1) + (sizeof(double) + sizeof(uint32_t)) *
			ctx->src_nhit);
	if (!m) return PSG_E_NOMEM;
	ctx->src_nray = nray;
	const SrcHits h = src_hits(ctx);
	cudaStream_t st = ctx->stream;
	PSG_CUDA(cudaMemcpyAsync((void *)h.off, ctx->scratch[S_OFFSETS].p, sizeof(int64_t) * (nray + 1),
			cudaMemcpyDeviceToDevice, st));
	if (tf.nhit) {
		PSG_CUDA(cudaMemcpyAsync((void *)h.ipar, ctx->scratch[S_HIT_IPAR].p, sizeof(uint32_t) * tf.nhit,
				cudaMemcpyDeviceToDevice, st));
		PSG_CUDA(cudaMemcpyAsync((void *)h.kern, ctx->scratch[S_HIT_KERN].p, sizeof(double) * tf.nhit,
				cudaMemcpyDeviceToDevice, st));
	}
	return PSG_OK;
}

// The traversal of a recombination tick: the emitted rays buf[R, R + *nlim)
// traversed (slabs from index 0), the source rays' counts from S_SRCHIT,
// then the scan and the offsets over all R + cap_rec rays.
int psg_trace_rec_fill_enqueue(psg_context *ctx, const psg_ray *buf, size_t R, size_t cap_rec, const unsigned *nlim,
		size_t cap, const PsgBatchDev *B) {
	cudaStream_t st = ctx->stream;
	const size_t nray = R + cap_rec;
	uint32_t *count = (uint32_t *)ctx->scratch[S_COUNT].p;
	unsigned long long *scan = count_scan(count, nray);
	int64_t *off64 = (int64_t *)ctx->scratch[S_OFFSETS].p;
	unsigned long long *d_max = ctx->d_counters + 4;
	unsigned long long *next_ray = ctx->d_counters + 9;
	const size_t scap = ctx->slab_cap;
	const size_t slots = cap_rec * scap;
	uint32_t *slab_ipar = (uint32_t *)ctx->scratch[S_REC_U32].p;
	double *slab_f64 = (double *)ctx->scratch[S_REC_F64].p;
	const int trw = std::max(1, std::min(TR_MAX_WARPS, ctx->tune.trace_warps));
	const size_t smem = sizeof(int) * (TR_STACK + 32 * (size_t)ctx->ppc + 32) * trw;
	const SrcHits h = src_hits(ctx);
	PSG_CUDA(cudaMemsetAsync(count, 0, sizeof(uint32_t) * (nray + 1), st));
	PSG_CUDA(cudaMemsetAsync(d_max, 0, 2 * sizeof(unsigned long long), st));
	PSG_CUDA(cudaMemsetAsync(next_ray, 0, sizeof(unsigned long long), st));
	k_trace_stack<<<ctx->trace_grid, 32 * trw, smem, st>>>(buf + R, cap_rec, ctx->d_wide_lo, ctx->d_wide_hi,
			ctx->d_leaf_psml, ctx->d_leaf_idx, ctx->ppc, count + R, scap, slab_ipar, slab_f64, slab_f64 + slots,
			next_ray, ctx->d_status, nlim);
	PSG_CHECK_LAUNCH();
	k_rec_counts<<<(unsigned)std::min<size_t>(blocks(nray, 256), 4 * (size_t)ctx->sms), 256, 0, st>>>(B, R, h.off,
			cap_rec, scap, count, ctx->d_counters + 3, ctx->d_status);
	PSG_CHECK_LAUNCH();
	PSG_CUDA(scan_enqueue(st, count, nray + 1, scan, (unsigned long long *)ctx->scratch[S_SCAN].p, Widen()));
	k_offsets64<<<blocks(nray + 1, 256), 256, 0, st>>>(scan, count, nray, off64, d_max, cap,
			ctx->d_counters + 24, ctx->d_status);
	PSG_CHECK_LAUNCH();
	ctx->launches += 5;
	return PSG_OK;
}

// The per-ray order of a recombination tick: the source rays' sorted hits
// copied from S_SRCHIT, the emitted rays (from R on) sorted from their slabs.
int psg_trace_rec_sort_enqueue(psg_context *ctx, size_t R, size_t nray, unsigned long long maxcount,
		const PsgBatchDev *B) {
	const SrcHits h = src_hits(ctx);
	k_copy_src_hits<<<blocks(R * 32, 256), 256, 0, ctx->stream>>>(B, R, h.off, h.ipar, h.kern,
			(const int64_t *)ctx->scratch[S_OFFSETS].p, (uint32_t *)ctx->scratch[S_HIT_IPAR].p,
			(double *)ctx->scratch[S_HIT_KERN].p);
	PSG_CHECK_LAUNCH();
	ctx->launches++;
	return psg_trace_sort_enqueue(ctx, nray, 0, maxcount, 1, R);
}

// Sizes the buffers psg_trace_rec_fill_enqueue uses for nray rays (allocates;
// before a capture) and its persistent grid.
int psg_trace_fill_prepare(psg_context *ctx, size_t nray) {
	const size_t scap = ctx->slab_cap;
	const size_t slots = nray * scap;
	if (!psg_scratch(ctx, S_COUNT, count_bytes(nray)) ||
			!psg_scratch(ctx, S_SCAN, sizeof(unsigned long long) * (scan_tiles(nray + 1) + 1)) ||
			!psg_scratch(ctx, S_OFFSETS, sizeof(int64_t) * (nray + 1) + 256) ||
			!psg_scratch(ctx, S_REC_U32, sizeof(uint32_t) * (slots ? slots : 1)) ||
			!psg_scratch(ctx, S_REC_F64, sizeof(double) * 2 * (slots ? slots : 1)))
		return PSG_E_NOMEM;
	const int trw = std::max(1, std::min(TR_MAX_WARPS, ctx->tune.trace_warps));
	const size_t smem = sizeof(int) * (TR_STACK + 32 * (size_t)ctx->ppc + 32) * trw;
	if (smem > 48 * 1024)
		PSG_CUDA(cudaFuncSetAttribute(k_trace_stack, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
	int per_sm = 1;
	PSG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_trace_stack, 32 * trw, smem));
	ctx->trace_grid = (unsigned)std::min<size_t>(blocks(nray, trw), (size_t)std::max(per_sm, 1) * ctx->sms);
	return PSG_OK;
}

// The traversal of nray device-resident rays into per-ray slabs, the hit
// counts' scan and the offsets (S_OFFSETS: int64 offsets[nray+1]). One host synchronisation reads the longest list,
// the status word and the hit total; a ray that outgrew its slab grows the
// slabs and reruns the traversal once.
int psg_trace_fill(psg_context *ctx, const psg_ray *d_rays, size_t nray, PsgTraceFill *tf) {
	if (!ctx->have_tree) return psg_fail(ctx, PSG_E_INVAL, "trace: no tree (psg_build_tree first)");
	cudaStream_t st = ctx->stream;
	uint32_t *count = (uint32_t *)psg_scratch(ctx, S_COUNT, count_bytes(nray));
	char *offmem = (char *)psg_scratch(ctx, S_OFFSETS, sizeof(int64_t) * (nray + 1) + 256);
	unsigned long long *tiles = (unsigned long long *)psg_scratch(ctx, S_SCAN,
			sizeof(unsigned long long) * (scan_tiles(nray + 1) + 1));
	if (!count || !offmem || !tiles) return PSG_E_NOMEM;
	unsigned long long *scan = count_scan(count, nray);
	int64_t *off64 = (int64_t *)offmem;
	unsigned long long *d_max = ctx->d_counters + 4;
	unsigned long long *next_ray = ctx->d_counters + 9;
	const int sms = ctx->sms;
	const int ppc = ctx->ppc;
	const int trw = std::max(1, std::min(TR_MAX_WARPS, ctx->tune.trace_warps));
	const size_t smem = sizeof(int) * (TR_STACK + 32 * (size_t)ppc + 32) * trw;
	if (smem > 48 * 1024)
		PSG_CUDA(cudaFuncSetAttribute(k_trace_stack, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
	size_t scap = 0;
	unsigned long long hdr[2] = {0, 0};      // longest list, hit total
	for (int attempt = 0; attempt < 2; attempt++) {
		scap = ctx->slab_cap ? ctx->slab_cap : 1024;
		const size_t slots = nray * scap;
		uint32_t *slab_ipar = (uint32_t *)psg_scratch(ctx, S_REC_U32, sizeof(uint32_t) * (slots ? slots : 1));
		double *slab_f64 = (double *)psg_scratch(ctx, S_REC_F64, sizeof(double) * 2 * (slots ? slots : 1));
		if (!slab_ipar || !slab_f64) return PSG_E_NOMEM;
		PSG_CUDA(cudaMemsetAsync(count + nray, 0, sizeof(uint32_t), st));
		PSG_CUDA(cudaMemsetAsync(d_max, 0, 2 * sizeof(unsigned long long), st));
		psg_mark_begin(ctx, PSG_K_TRACE_FILL);
		if (nray) {
			PSG_CUDA(cudaMemsetAsync(next_ray, 0, sizeof(unsigned long long), st));
			int per_sm = 1;
			PSG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_trace_stack, 32 * trw, smem));
			const unsigned tgrid = (unsigned)std::min<size_t>(blocks(nray, trw), (size_t)std::max(per_sm, 1) * sms);
			k_trace_stack<<<tgrid, 32 * trw, smem, st>>>(d_rays, nray, ctx->d_wide_lo,
					ctx->d_wide_hi, ctx->d_leaf_psml, ctx->d_leaf_idx, ppc, count, scap, slab_ipar,
					slab_f64, slab_f64 + slots, next_ray, ctx->d_status, nullptr);
			ctx->launches++;
		}
		PSG_CHECK_LAUNCH();
		psg_mark_end(ctx);
		PSG_CUDA(scan_enqueue(st, count, nray + 1, scan, tiles, Widen()));
		k_offsets64<<<blocks(nray + 1, 256), 256, 0, st>>>(scan, count, nray, off64, d_max, 0, nullptr,
				nullptr);
		PSG_CHECK_LAUNCH();
		ctx->launches++;
		PSG_CUDA(cudaMemcpyAsync(hdr, d_max, sizeof(hdr), cudaMemcpyDeviceToHost, st));
		uint32_t stw = 0;
		PSG_CUDA(cudaMemcpyAsync(&stw, ctx->d_status, sizeof(stw), cudaMemcpyDeviceToHost, st));
		PSG_CUDA(cudaStreamSynchronize(st));
		ctx->host_syncs++;
		if (stw & PSG_ST_STACK) {
			PSG_CUDA(cudaMemsetAsync(ctx->d_status, 0, sizeof(uint32_t), st));
			return psg_fail(ctx, PSG_E_OVERFLOW, "trace: traversal stack overflow (tree deeper than supported)");
		}
		if (hdr[0] <= scap) break;
		size_t want = 1024;
		while (want < hdr[0] + hdr[0] / 4) want <<= 1;
		ctx->slab_cap = want;
		if (attempt == 1) return psg_fail(ctx, PSG_E_OVERFLOW, "trace: hit lists grew between passes");
	}
	if (!ctx->slab_cap) ctx->slab_cap = scap;
	if (hdr[1] >= (unsigned long long)INT32_MAX)
		return psg_fail(ctx, PSG_E_OVERFLOW, "trace: %llu hits in one batch exceed 2^31", hdr[1]);
	tf->nhit = (size_t)hdr[1];
	tf->maxcount = hdr[0];
	tf->scap = scap;
	return PSG_OK;
}

// Buffers of the sorted hit lists for up to cap hits: S_HIT_IPAR, S_RAW_D
// (sorted d at + cap), S_HIT_KERN (b, or the column-density factor), and
// the class lists. Allocates; call before a stream capture.
int psg_trace_sort_prepare(psg_context *ctx, size_t nray, size_t cap, unsigned long long maxcount) {
	const size_t hb = cap ? cap : 1;
	uint32_t *hit_ipar = (uint32_t *)psg_scratch(ctx, S_HIT_IPAR, sizeof(uint32_t) * hb);
	double *hit_db = (double *)psg_scratch(ctx, S_RAW_D, sizeof(double) * 2 * hb);
	double *hit_b = (double *)psg_scratch(ctx, S_HIT_KERN, sizeof(double) * hb);
	uint32_t *lists = (uint32_t *)psg_scratch(ctx, S_RAYLIST, sizeof(uint32_t) * (SORT_NCLS + 1) * (nray + 1));
	if (!hit_ipar || !hit_db || !hit_b || !lists) return PSG_E_NOMEM;
	ctx->hit_cap = hb;
	// the long rays' two halves of (d, key) pairs, at their list offsets
	if (maxcount > PSG_SORT_MAX && !psg_scratch(ctx, S_KEYS, sizeof(LongHit) * 2 * hb)) return PSG_E_NOMEM;
	// shared-memory limits and resident blocks per multiprocessor of the
	// eight class kernels (their persistent grids), once per context
	if (!ctx->sort_grid[0]) {
		int c = 0;
#define PSG_SORT_ATTR(T, I)                                                                                    \
	{                                                                                                        \
		if (sort_smem_bytes<T, I>() > 48 * 1024)                                                             \
			PSG_CUDA(cudaFuncSetAttribute(k_sort_block<T, I>, cudaFuncAttributeMaxDynamicSharedMemorySize,    \
					(int)sort_smem_bytes<T, I>()));                                                          \
		int per_sm = 1;                                                                                      \
		PSG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sort_block<T, I>, T,               \
				sort_smem_bytes<T, I>()));                                                                   \
		ctx->sort_grid[c++] = (unsigned)std::max(per_sm, 1) * (unsigned)ctx->sms;                             \
	}
		PSG_SORT_ATTR(32, 2) PSG_SORT_ATTR(32, 4) PSG_SORT_ATTR(64, 4) PSG_SORT_ATTR(128, 4)
		PSG_SORT_ATTR(128, 8) PSG_SORT_ATTR(256, 8) PSG_SORT_ATTR(256, 16) PSG_SORT_ATTR(512, 16)
#undef PSG_SORT_ATTR
	}
	return PSG_OK;
}

// The size classes a call with lists up to maxcount long can fill.
int psg_sort_classes(unsigned long long maxcount) {
	static const unsigned long long lower[SORT_NCLS] = {0, 64, 128, 256, 512, 1024, 2048, 4096};
	int c = 0;
	while (c < SORT_NCLS && maxcount > lower[c]) c++;
	return c;
}

// The per-ray sort by (d, ipar) of the filled slabs into the CSR lists.
// Launch sizes are fixed by nray (the persistent class kernels read their
// ray counts on the device), so it can be captured in a graph; with
// maxcount above PSG_SORT_MAX the long rays' kernel runs too.
int psg_trace_sort_enqueue(psg_context *ctx, size_t nray, size_t nhit, unsigned long long maxcount,
		int want_kern, size_t r0) {
	(void)nhit;
	cudaStream_t st = ctx->stream;
	const size_t hb = ctx->hit_cap;
	const size_t scap = ctx->slab_cap;
	const size_t slots = (nray - r0) * scap;
	int64_t *off64 = (int64_t *)ctx->scratch[S_OFFSETS].p;
	uint32_t *hit_ipar = (uint32_t *)ctx->scratch[S_HIT_IPAR].p;
	double *hit_d = (double *)ctx->scratch[S_RAW_D].p + hb;
	double *hit_b = (double *)ctx->scratch[S_HIT_KERN].p;
	uint32_t *slab_ipar = (uint32_t *)ctx->scratch[S_REC_U32].p;
	double *slab_d = (double *)ctx->scratch[S_REC_F64].p;
	double *slab_b = slab_d + slots;
	if (nray <= r0) return PSG_OK;
	psg_mark_begin(ctx, PSG_K_SORT);
	{
		uint32_t *lists = (uint32_t *)ctx->scratch[S_RAYLIST].p;
		unsigned long long *d_ncls = ctx->d_counters + 16, *d_nlong = ctx->d_counters + 25;
		PSG_CUDA(cudaMemsetAsync(d_ncls, 0, SORT_NCLS * sizeof(unsigned long long), st));
		PSG_CUDA(cudaMemsetAsync(d_nlong, 0, sizeof(unsigned long long), st));
		k_sort_classify<<<blocks(nray - r0, 256), 256, 0, st>>>(r0, nray, off64, lists, nray + 1, d_ncls, d_nlong);
		PSG_CHECK_LAUNCH();
		const PhysParams PP = psg_phys_params(ctx);
		const size_t stride = nray + 1;
		// a class whose rays all have more hits than the call's longest list
		// is empty: not launched (psg_sort_classes; part of a graph's key)
		const int ncls = psg_sort_classes(maxcount);
		auto launch_block = [&](auto kern, int tpr, size_t smem, int c) -> int {
			if (c >= ncls) return PSG_OK;
			const unsigned grid = (unsigned)std::min<size_t>(nray - r0, (size_t)ctx->sort_grid[c]);
			kern<<<grid, tpr, smem, st>>>(lists + c * stride, d_ncls + c, off64, scap, slab_ipar, slab_d,
					slab_b, hit_ipar, hit_d, hit_b, want_kern, ctx->d_psml, PP, ctx->d_order, r0);
			PSG_CHECK_LAUNCH();
			ctx->launches++;
			return PSG_OK;
		};
		int rcs = launch_block(k_sort_block<32, 2>, 32, sort_smem_bytes<32, 2>(), 0);
		if (!rcs) rcs = launch_block(k_sort_block<32, 4>, 32, sort_smem_bytes<32, 4>(), 1);
		if (!rcs) rcs = launch_block(k_sort_block<64, 4>, 64, sort_smem_bytes<64, 4>(), 2);
		if (!rcs) rcs = launch_block(k_sort_block<128, 4>, 128, sort_smem_bytes<128, 4>(), 3);
		if (!rcs) rcs = launch_block(k_sort_block<128, 8>, 128, sort_smem_bytes<128, 8>(), 4);
		if (!rcs) rcs = launch_block(k_sort_block<256, 8>, 256, sort_smem_bytes<256, 8>(), 5);
		if (!rcs) rcs = launch_block(k_sort_block<256, 16>, 256, sort_smem_bytes<256, 16>(), 6);
		if (!rcs) rcs = launch_block(k_sort_block<512, 16>, 512, sort_smem_bytes<512, 16>(), 7);
		if (rcs) return rcs;
		ctx->launches++;
		if (maxcount > PSG_SORT_MAX) {
			// rays longer than the shared-memory classes: a block each
			const unsigned grid = (unsigned)std::min<size_t>(nray - r0, (size_t)ctx->sms);
			k_sort_long<<<grid, LONG_NT, 0, st>>>(lists + SORT_NCLS * stride, d_nlong, off64, scap, slab_ipar,
					slab_d, slab_b, hit_ipar, hit_d, hit_b, want_kern, ctx->d_psml, PP, ctx->d_order,
					(LongHit *)ctx->scratch[S_KEYS].p, hb, r0);
			PSG_CHECK_LAUNCH();
			ctx->launches++;
		}
	}
	psg_mark_end(ctx);
	return PSG_OK;
}

// Traces nray device-resident rays: fill, buffers sized to the hits, sort.
// Leaves in scratch: S_OFFSETS, S_HIT_IPAR (sorted leaf-order indices),
// S_RAW_D (sorted d at + hit_cap) and S_HIT_KERN (sorted b, or with
// want_kern the column-density factor).
int psg_trace_internal(psg_context *ctx, const psg_ray *d_rays, size_t nray, int want_kern) {
	PsgTraceFill tf;
	int rc = psg_trace_fill(ctx, d_rays, nray, &tf);
	if (rc) return rc;
	rc = psg_trace_sort_prepare(ctx, nray, tf.nhit, tf.maxcount);
	if (rc) return rc;
	return psg_trace_sort_enqueue(ctx, nray, tf.nhit, tf.maxcount, want_kern, 0);
}

__global__ void k_caller_index(size_t n, const uint32_t *__restrict__ in, const uint32_t *__restrict__ order,
		uint32_t *__restrict__ out) {
	const size_t h = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
	if (h < n) out[h] = order[in[h]];
}

// copies the traced hit lists to host Xtype records
static int download_hits(psg_context *ctx, size_t nray, int64_t *offsets, psg_xtype **x, size_t *size,
		size_t *nhit_out) {
	cudaStream_t st = ctx->stream;
	int64_t *off64 = (int64_t *)ctx->scratch[S_OFFSETS].p;
	std::vector<int64_t> off(nray + 1);
	PSG_CUDA(cudaMemcpyAsync(off.data(), off64, sizeof(int64_t) * (nray + 1), cudaMemcpyDeviceToHost, st));
	PSG_CUDA(cudaStreamSynchronize(st));
	const size_t nhit = (size_t)off[nray];
	if (offsets) memcpy(offsets, off.data(), sizeof(int64_t) * (nray + 1));
	if (*x == nullptr || *size < nhit) {
		size_t want = *size ? *size : 1000;
		while (want < nhit) want *= 2;
		psg_xtype *nx = (psg_xtype *)realloc(*x, sizeof(psg_xtype) * want);
		if (!nx) return psg_fail(ctx, PSG_E_NOMEM, "trace: host allocation failed");
		*x = nx;
		*size = want;
	}
	if (nhit) {
		std::vector<uint32_t> ip(nhit);
		std::vector<double> d(nhit), b(nhit);
		double *hit_d = (double *)ctx->scratch[S_RAW_D].p + ctx->hit_cap;
		// hits carry internal particle positions: the caller's indices
		const uint32_t *hit_ipar = (const uint32_t *)ctx->scratch[S_HIT_IPAR].p;
		if (ctx->d_order) {
			uint32_t *mapped = (uint32_t *)psg_scratch(ctx, S_MAP, sizeof(uint32_t) * nhit);
			if (!mapped) return PSG_E_NOMEM;
			k_caller_index<<<(unsigned)((nhit + 255) / 256), 256, 0, st>>>(nhit, hit_ipar, ctx->d_order, mapped);
			PSG_CHECK_LAUNCH();
			hit_ipar = mapped;
		}
		PSG_CUDA(cudaMemcpyAsync(ip.data(), hit_ipar, sizeof(uint32_t) * nhit, cudaMemcpyDeviceToHost, st));
		PSG_CUDA(cudaMemcpyAsync(d.data(), hit_d, sizeof(double) * nhit, cudaMemcpyDeviceToHost, st));
		PSG_CUDA(cudaMemcpyAsync(b.data(), ctx->scratch[S_HIT_KERN].p, sizeof(double) * nhit, cudaMemcpyDeviceToHost, st));
		PSG_CUDA(cudaStreamSynchronize(st));
		for (size_t h = 0; h < nhit; h++) {
			(*x)[h].ipar = ip[h];
			(*x)[h].d = d[h];
			(*x)[h].b = b[h];
		}
	}
	*nhit_out = nhit;
	return PSG_OK;
}

static int upload_rays(psg_context *ctx, const psg_ray *rays, size_t nray, psg_ray **d_rays) {
	psg_ray *d = (psg_ray *)psg_scratch(ctx, S_RAYS, sizeof(psg_ray) * (nray ? nray : 1));
	if (!d) return PSG_E_NOMEM;
	if (nray) PSG_CUDA(cudaMemcpyAsync(d, rays, sizeof(psg_ray) * nray, cudaMemcpyHostToDevice, ctx->stream));
	*d_rays = d;
	return PSG_OK;
}

extern "C" int psg_trace(psg_context *ctx, const psg_ray *rays, size_t nray, int64_t *offsets,
		psg_xtype **x, size_t *size) {
	if (!ctx) return PSG_E_INVAL;
	if ((nray && !rays) || !x || !size) return psg_fail(ctx, PSG_E_INVAL, "psg_trace: null argument");
	PSG_CUDA(cudaSetDevice(ctx->device));
	psg_ray *d_rays = nullptr;
	int rc = upload_rays(ctx, rays, nray, &d_rays);
	if (rc) return rc;
	rc = psg_trace_internal(ctx, d_rays, nray, 0);
	if (rc) return rc;
	size_t nhit = 0;
	return download_hits(ctx, nray, offsets, x, size, &nhit);
}

extern "C" size_t psg_rt_trace(psg_context *ctx, const float s[3], const float dir[3], const float dist,
		psg_xtype **x, size_t *size) {
	if (!ctx || !s || !dir || !x || !size) return (size_t)-1;
	psg_ray ray;
	memset(&ray, 0, sizeof(ray));
	for (int d = 0; d < 3; d++) { ray.s[d] = s[d]; ray.dir[d] = dir[d]; }
	ray.length = dist;
	if (cudaSetDevice(ctx->device) != cudaSuccess) return (size_t)-1;
	psg_ray *d_rays = nullptr;
	if (upload_rays(ctx, &ray, 1, &d_rays)) return (size_t)-1;
	if (psg_trace_internal(ctx, d_rays, 1, 0)) return (size_t)-1;
	size_t nhit = 0;
	if (download_hits(ctx, 1, nullptr, x, size, &nhit)) return (size_t)-1;
	return nhit;
}
