// Octree built on the device; replaces rt_switch_epoch() raytrace.c:41-151.
//
// The reference inserts particles one at a time into a region octree and
// splits a leaf when a particle arrives while it holds ppc particles. The
// resulting tree does not depend on insertion order: a cell is split exactly
// when its region holds more than ppc particles. So the tree is rebuilt here
// without insertion:
//   1. every particle gets a 63-bit key, 3 bits per level, by descending the
//      region octree with the reference's own float arithmetic (the split
//      point of a cell is fl(top+bot)*0.5, split() raytrace.c:279-281, and a
//      particle is in the upper child iff pos >= split point, inside()
//      raytrace.c:306-317);
//   2. keys are radix sorted, so every cell's particles are one contiguous
//      run and runs appear in depth-first order with children 0..7;
//   3. cells are created level by level from the runs (a cell with more than
//      ppc particles gets 8 children, empty ones included);
//   4. boxes are recomputed bottom-up as the reference does (raytrace.c:
//      100-150): a leaf's box is the min/max of pos -+ sml of its particles,
//      an empty leaf keeps its region, a parent is the union of its 8
//      children;
//   5. cells are written in depth-first order with, per cell, the index just
//      past its subtree (a skip pointer) and the first particle of its run,
//      which is the layout the stackless traversal reads.
#include <cub/cub.cuh>

#include <string.h>

#include <vector>

#include "psg_internal.cuh"

namespace {

__global__ void k_keys(size_t n, const float4 *__restrict__ psml, float box,
		unsigned long long *__restrict__ keys, uint32_t *__restrict__ vals) {
	const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
	if (i >= n) return;
	const float4 p = psml[i];
	const float pv[3] = {p.x, p.y, p.z};
	bool inside = true;
	for (int d = 0; d < 3; d++) inside &= !(pv[d] >= box || pv[d] < 0.0f);
	unsigned long long key = PSG_KEY_OUTSIDE;
	if (inside) {
		float lo[3] = {0.0f, 0.0f, 0.0f}, hi[3] = {box, box, box};
		key = 0;
		for (int l = 0; l < PSG_MAX_LEVELS; l++) {
			unsigned k = 0;
			for (int d = 0; d < 3; d++) {
				const float mid = rn_fmul(rn_fadd(hi[d], lo[d]), 0.5f);
				const bool up = pv[d] >= mid;
				if (up) lo[d] = mid; else hi[d] = mid;
				k |= (unsigned)up << d;
			}
			key = (key << 3) | k;
		}
	}
	keys[i] = key;
	vals[i] = (uint32_t)i;
}

__global__ void k_count_valid(size_t n, const unsigned long long *__restrict__ keys,
		unsigned long long *out) {
	// first index whose key is the outside marker (keys sorted ascending)
	size_t lo = 0, hi = n;
	while (lo < hi) {
		const size_t mid = (lo + hi) / 2;
		if (keys[mid] == PSG_KEY_OUTSIDE) hi = mid; else lo = mid + 1;
	}
	*out = lo;
}

// Internal cells per level: position i starts a run of equal level-L
// prefixes longer than ppc iff keys[i-1] has another prefix and keys[i+ppc]
// the same one. Level 0 is the root (empty prefix).
__global__ void k_count_internal(const unsigned long long *__restrict__ keys, uint32_t nvalid,
		int ppc, unsigned long long *__restrict__ count) {
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= nvalid) return;
	const unsigned long long k = keys[i];
	const bool has_prev = i > 0;
	const unsigned long long kp = has_prev ? keys[i - 1] : 0ull;
	const bool has_far = (uint64_t)i + ppc < nvalid;
	const unsigned long long kf = has_far ? keys[i + ppc] : 0ull;
	for (int l = 0; l <= PSG_MAX_LEVELS; l++) {
		const int shift = 3 * (PSG_MAX_LEVELS - l);
		const unsigned long long pk = shift >= 63 ? 0ull : (k >> shift);
		const bool starts = !has_prev || (shift >= 63 ? false : ((kp >> shift) != pk));
		const bool big = has_far && (shift >= 63 ? true : ((kf >> shift) == pk));
		if (starts && big) atomicAdd(&count[l], 1ull);
	}
}

struct Cells {
	uint32_t *start, *end;
	float4 *lo, *hi;       // region box while expanding, then the AABB
	int32_t *parent, *fchild, *size, *pre;
	int32_t *flag;         // scratch: child is internal
};

__global__ void k_init_root(Cells c, uint32_t nvalid, float box) {
	c.start[0] = 0;
	c.end[0] = nvalid;
	c.lo[0] = make_float4(0.f, 0.f, 0.f, 0.f);
	c.hi[0] = make_float4(box, box, box, 0.f);
	c.parent[0] = -1;
	c.fchild[0] = -1;
}

// Create the 8 children of every cell in the frontier (cells of `level` that
// hold more than ppc particles).
__global__ void k_expand(Cells c, const int32_t *__restrict__ frontier, int nfront, int level,
		int base, int ppc, const unsigned long long *__restrict__ keys) {
	const int f = blockIdx.x * blockDim.x + threadIdx.x;
	if (f >= nfront) return;
	const int cell = frontier[f];
	const uint32_t s = c.start[cell], e = c.end[cell];
	const int shift = 3 * (PSG_MAX_LEVELS - 1 - level);
	uint32_t bound[9];
	bound[0] = s;
	bound[8] = e;
	for (unsigned k = 1; k < 8; k++) {
		uint32_t lo = bound[k - 1], hi = e;
		while (lo < hi) {
			const uint32_t mid = lo + (hi - lo) / 2;
			if (((keys[mid] >> shift) & 7ull) < k) lo = mid + 1; else hi = mid;
		}
		bound[k] = lo;
	}
	const float4 rlo = c.lo[cell], rhi = c.hi[cell];
	const float mid[3] = {rn_fmul(rn_fadd(rhi.x, rlo.x), 0.5f), rn_fmul(rn_fadd(rhi.y, rlo.y), 0.5f),
		rn_fmul(rn_fadd(rhi.z, rlo.z), 0.5f)};
	const float lo3[3] = {rlo.x, rlo.y, rlo.z}, hi3[3] = {rhi.x, rhi.y, rhi.z};
	const int first = base + 8 * f;
	c.fchild[cell] = first;
	for (int k = 0; k < 8; k++) {
		float clo[3], chi[3];
		for (int d = 0; d < 3; d++) {
			const bool up = (k >> d) & 1;
			clo[d] = up ? mid[d] : lo3[d];
			chi[d] = up ? hi3[d] : mid[d];
		}
		const int ch = first + k;
		c.start[ch] = bound[k];
		c.end[ch] = bound[k + 1];
		c.lo[ch] = make_float4(clo[0], clo[1], clo[2], 0.f);
		c.hi[ch] = make_float4(chi[0], chi[1], chi[2], 0.f);
		c.parent[ch] = cell;
		c.fchild[ch] = -1;
		c.flag[ch - base] = (bound[k + 1] - bound[k]) > (uint32_t)ppc;
	}
}

__global__ void k_compact(const int32_t *__restrict__ flag, const int32_t *__restrict__ scan,
		int nchild, int base, int32_t *__restrict__ next) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= nchild) return;
	if (flag[i]) next[scan[i]] = base + i;
}

// Bottom-up: subtree sizes and boxes for the cells [b, e) of one level.
__global__ void k_bottom_up(Cells c, int b, int e, const float4 *__restrict__ lpsml) {
	const int cell = b + blockIdx.x * blockDim.x + threadIdx.x;
	if (cell >= e) return;
	const int fc = c.fchild[cell];
	if (fc < 0) {
		c.size[cell] = 1;
		const uint32_t s = c.start[cell], t = c.end[cell];
		if (t > s) {
			float lo[3], hi[3];
			for (uint32_t p = s; p < t; p++) {
				const float4 q = lpsml[p];
				const float v[3] = {q.x, q.y, q.z};
				for (int d = 0; d < 3; d++) {
					const float a = rn_fsub(v[d], q.w), z = rn_fadd(v[d], q.w);
					if (p == s || a < lo[d]) lo[d] = a;
					if (p == s || z > hi[d]) hi[d] = z;
				}
			}
			c.lo[cell] = make_float4(lo[0], lo[1], lo[2], 0.f);
			c.hi[cell] = make_float4(hi[0], hi[1], hi[2], 0.f);
		}
	} else {
		int sz = 1;
		float lo[3], hi[3];
		for (int k = 0; k < 8; k++) {
			sz += c.size[fc + k];
			const float4 a = c.lo[fc + k], z = c.hi[fc + k];
			const float av[3] = {a.x, a.y, a.z}, zv[3] = {z.x, z.y, z.z};
			for (int d = 0; d < 3; d++) {
				if (k == 0 || av[d] < lo[d]) lo[d] = av[d];
				if (k == 0 || zv[d] > hi[d]) hi[d] = zv[d];
			}
		}
		c.size[cell] = sz;
		c.lo[cell] = make_float4(lo[0], lo[1], lo[2], 0.f);
		c.hi[cell] = make_float4(hi[0], hi[1], hi[2], 0.f);
	}
}

// Top-down: depth-first index of the children of internal cells [b, e).
__global__ void k_preorder(Cells c, int b, int e) {
	const int cell = b + blockIdx.x * blockDim.x + threadIdx.x;
	if (cell >= e) return;
	const int fc = c.fchild[cell];
	if (fc < 0) return;
	int run = c.pre[cell] + 1;
	for (int k = 0; k < 8; k++) {
		c.pre[fc + k] = run;
		run += c.size[fc + k];
	}
}

__global__ void k_emit(Cells c, int ncell, uint32_t nvalid, float4 *__restrict__ out_lo,
		float4 *__restrict__ out_hi) {
	const int cell = blockIdx.x * blockDim.x + threadIdx.x;
	if (cell > ncell) return;
	if (cell == ncell) {     // sentinel: closes the particle run of the last cell
		out_lo[ncell] = make_float4(0.f, 0.f, 0.f, __int_as_float(ncell + 1));
		out_hi[ncell] = make_float4(0.f, 0.f, 0.f, __int_as_float((int)nvalid));
		return;
	}
	const int i = c.pre[cell];
	const float4 a = c.lo[cell], z = c.hi[cell];
	out_lo[i] = make_float4(a.x, a.y, a.z, __int_as_float(i + c.size[cell]));
	out_hi[i] = make_float4(z.x, z.y, z.z, __int_as_float((int)c.start[cell]));
}

// Level-order layout for the stack traversal: cells as built, the 8 children
// of a cell contiguous. lo.w = index of the first child, or -1-count for a
// leaf of `count` particles; hi.w = first particle of the cell (leaf order).
__global__ void k_emit_wide(Cells c, int ncell, float4 *__restrict__ out_lo, float4 *__restrict__ out_hi) {
	const int cell = blockIdx.x * blockDim.x + threadIdx.x;
	if (cell >= ncell) return;
	const float4 a = c.lo[cell], z = c.hi[cell];
	const int fc = c.fchild[cell];
	const int w = fc >= 0 ? fc : -1 - (int)(c.end[cell] - c.start[cell]);
	out_lo[cell] = make_float4(a.x, a.y, a.z, __int_as_float(w));
	out_hi[cell] = make_float4(z.x, z.y, z.z, __int_as_float((int)c.start[cell]));
}

// The traversal's copy of the particles in the box (the first nvalid of the
// leaf order, which the particle arrays are already in) and their index,
// marked when flagged PF_INVALID (psystem.h:28).
__global__ void k_gather_particles(size_t nvalid, const float4 *__restrict__ psml, const int8_t *__restrict__ flag,
		float4 *__restrict__ lpsml, uint32_t *__restrict__ lidx) {
	const size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
	if (k >= nvalid) return;
	lpsml[k] = psml[k];
	lidx[k] = (uint32_t)k | ((flag[k] & 1) ? PSG_INVALID_BIT : 0u);
}

inline unsigned blocks(size_t n, int bs) { return (unsigned)((n + bs - 1) / bs); }

}  // namespace

extern "C" int psg_build_tree(psg_context *ctx, int ppc) {
	if (!ctx) return PSG_E_INVAL;
	if (!ctx->n) return psg_fail(ctx, PSG_E_INVAL, "psg_build_tree: no particles loaded");
	if (ppc < 1 || ppc > 255) return psg_fail(ctx, PSG_E_INVAL, "psg_build_tree: ppc must be in 1..255");
	PSG_CUDA(cudaSetDevice(ctx->device));
	cudaStream_t st = ctx->stream;
	const size_t n = ctx->n;
	const float box = (float)ctx->boxsize;

	// 1-2: keys and sort
	unsigned long long *keys = (unsigned long long *)psg_scratch(ctx, S_KEYS, sizeof(unsigned long long) * 2 * n);
	uint32_t *vals = (uint32_t *)psg_scratch(ctx, S_VALS, sizeof(uint32_t) * 2 * n);
	if (!keys || !vals) return PSG_E_NOMEM;
	unsigned long long *keys_s = keys + n;
	uint32_t *vals_s = vals + n;
	k_keys<<<blocks(n, 256), 256, 0, st>>>(n, ctx->d_psml, box, keys, vals);
	PSG_CHECK_LAUNCH();
	size_t tmp = 0;
	PSG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, keys, keys_s, vals, vals_s, (int64_t)n, 0, 64, st));
	void *d_tmp = psg_scratch(ctx, S_CUB, tmp);
	if (!d_tmp) return PSG_E_NOMEM;
	PSG_CUDA(cub::DeviceRadixSort::SortPairs(d_tmp, tmp, keys, keys_s, vals, vals_s, (int64_t)n, 0, 64, st));
	unsigned long long *d_nvalid = (unsigned long long *)psg_scratch(ctx, S_COUNT, 64);
	if (!d_nvalid) return PSG_E_NOMEM;
	k_count_valid<<<1, 1, 0, st>>>(n, keys_s, d_nvalid);
	PSG_CHECK_LAUNCH();
	unsigned long long nvalid = 0;
	PSG_CUDA(cudaMemcpyAsync(&nvalid, d_nvalid, sizeof(nvalid), cudaMemcpyDeviceToHost, st));
	PSG_CUDA(cudaStreamSynchronize(st));

	// every per-particle array into the leaf order of this tree (vals_s
	// holds the current positions sorted by key, the particles outside the
	// box last)
	int prc = psg_permute_particles(ctx, vals_s);
	if (prc) return prc;

	// particles in leaf order
	if (ctx->d_leaf_psml) cudaFree(ctx->d_leaf_psml);
	if (ctx->d_leaf_idx) cudaFree(ctx->d_leaf_idx);
	ctx->d_leaf_psml = nullptr;
	ctx->d_leaf_idx = nullptr;
	ctx->have_tree = 0;
	PSG_CUDA(cudaMalloc(&ctx->d_leaf_psml, sizeof(float4) * (nvalid + 1)));
	PSG_CUDA(cudaMalloc(&ctx->d_leaf_idx, sizeof(uint32_t) * (nvalid + 1)));
	if (nvalid)
		k_gather_particles<<<blocks(nvalid, 256), 256, 0, st>>>(nvalid, ctx->d_psml, ctx->d_flag,
				ctx->d_leaf_psml, ctx->d_leaf_idx);
	PSG_CHECK_LAUNCH();

	// 3: cells level by level. A run of more than ppc equal level-L prefixes
	// is exactly an internal cell of level L; counting them first sizes the
	// cell arrays exactly.
	unsigned long long *d_levels = (unsigned long long *)psg_scratch(ctx, S_COUNT, 64 * sizeof(unsigned long long));
	if (!d_levels) return PSG_E_NOMEM;
	PSG_CUDA(cudaMemsetAsync(d_levels, 0, 64 * sizeof(unsigned long long), st));
	if (nvalid)
		k_count_internal<<<blocks(nvalid, 256), 256, 0, st>>>(keys_s, (uint32_t)nvalid, ppc, d_levels);
	PSG_CHECK_LAUNCH();
	unsigned long long internal[PSG_MAX_LEVELS + 1];
	PSG_CUDA(cudaMemcpyAsync(internal, d_levels, sizeof(internal), cudaMemcpyDeviceToHost, st));
	PSG_CUDA(cudaStreamSynchronize(st));
	if (internal[PSG_MAX_LEVELS])
		return psg_fail(ctx, PSG_E_OVERFLOW,
				"psg_build_tree: more than %d particles share a cell at depth %d", ppc, PSG_MAX_LEVELS);
	size_t total_internal = 0;
	for (int l = 0; l < PSG_MAX_LEVELS; l++) total_internal += internal[l];
	const size_t cap = 1 + 8 * total_internal;
	if (cap >= (size_t)INT32_MAX)
		return psg_fail(ctx, PSG_E_OVERFLOW, "psg_build_tree: %zu cells exceed the 32-bit index", cap);
	size_t maxfront = 1;
	for (int l = 0; l < PSG_MAX_LEVELS; l++) maxfront = internal[l] > maxfront ? internal[l] : maxfront;
	Cells c{};
	int32_t *front = nullptr, *front_next = nullptr, *scan = nullptr;
	{
		const size_t bytes = cap * (2 * sizeof(float4) + 7 * sizeof(int32_t)) + 8 * maxfront * sizeof(int32_t)
			+ 2 * maxfront * sizeof(int32_t) + 16 * 256;
		char *m = (char *)psg_scratch(ctx, S_TREE, bytes);
		if (!m) return PSG_E_NOMEM;
		size_t off = 0;
		auto take = [&](size_t b) { char *q = m + off; off += (b + 255) & ~(size_t)255; return q; };
		c.lo = (float4 *)take(sizeof(float4) * cap);
		c.hi = (float4 *)take(sizeof(float4) * cap);
		c.start = (uint32_t *)take(sizeof(uint32_t) * cap);
		c.end = (uint32_t *)take(sizeof(uint32_t) * cap);
		c.parent = (int32_t *)take(sizeof(int32_t) * cap);
		c.fchild = (int32_t *)take(sizeof(int32_t) * cap);
		c.size = (int32_t *)take(sizeof(int32_t) * cap);
		c.pre = (int32_t *)take(sizeof(int32_t) * cap);
		c.flag = (int32_t *)take(sizeof(int32_t) * 8 * maxfront);
		scan = (int32_t *)take(sizeof(int32_t) * 8 * maxfront);
		front = (int32_t *)take(sizeof(int32_t) * maxfront);
		front_next = (int32_t *)take(sizeof(int32_t) * maxfront);
	}
	k_init_root<<<1, 1, 0, st>>>(c, (uint32_t)nvalid, box);
	PSG_CHECK_LAUNCH();
	std::vector<int> level_begin{0}, level_end{1};
	size_t ncell = 1;
	PSG_CUDA(cudaMemsetAsync(front, 0, sizeof(int32_t), st));
	for (int level = 0; level < PSG_MAX_LEVELS && internal[level] > 0; level++) {
		const int nfront = (int)internal[level];
		const size_t nchild = (size_t)nfront * 8;
		const int base = (int)ncell;
		k_expand<<<blocks(nfront, 128), 128, 0, st>>>(c, front, nfront, level, base, ppc, keys_s);
		PSG_CHECK_LAUNCH();
		size_t stmp = 0;
		PSG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, stmp, c.flag, scan, (int)nchild, st));
		void *dt = psg_scratch(ctx, S_CUB, stmp);
		if (!dt) return PSG_E_NOMEM;
		PSG_CUDA(cub::DeviceScan::ExclusiveSum(dt, stmp, c.flag, scan, (int)nchild, st));
		k_compact<<<blocks(nchild, 256), 256, 0, st>>>(c.flag, scan, (int)nchild, base, front_next);
		PSG_CHECK_LAUNCH();
		int last_scan = 0, last_flag = 0;
		PSG_CUDA(cudaMemcpyAsync(&last_scan, scan + nchild - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
		PSG_CUDA(cudaMemcpyAsync(&last_flag, c.flag + nchild - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
		PSG_CUDA(cudaStreamSynchronize(st));
		const unsigned long long want = level + 1 < PSG_MAX_LEVELS ? internal[level + 1] : 0ull;
		if ((unsigned long long)(last_scan + last_flag) != want)
			return psg_fail(ctx, PSG_E_CUDA, "psg_build_tree: level %d has %d internal cells, expected %llu",
					level + 1, last_scan + last_flag, want);
		ncell += nchild;
		level_begin.push_back(base);
		level_end.push_back((int)ncell);
		std::swap(front, front_next);
	}
	if (ncell != cap)
		return psg_fail(ctx, PSG_E_CUDA, "psg_build_tree: built %zu cells, expected %zu", ncell, cap);
	const int nlevels = (int)level_begin.size();

	// 4: bottom-up sizes and boxes
	for (int l = nlevels - 1; l >= 0; l--) {
		const int b = level_begin[l], e = level_end[l];
		k_bottom_up<<<blocks(e - b, 128), 128, 0, st>>>(c, b, e, ctx->d_leaf_psml);
		PSG_CHECK_LAUNCH();
	}
	// 5: depth-first numbering and output
	PSG_CUDA(cudaMemsetAsync(c.pre, 0, sizeof(int32_t), st));
	for (int l = 0; l < nlevels - 1; l++) {
		const int b = level_begin[l], e = level_end[l];
		k_preorder<<<blocks(e - b, 128), 128, 0, st>>>(c, b, e);
		PSG_CHECK_LAUNCH();
	}
	if (ctx->d_cell_lo) cudaFree(ctx->d_cell_lo);
	if (ctx->d_cell_hi) cudaFree(ctx->d_cell_hi);
	ctx->d_cell_lo = ctx->d_cell_hi = nullptr;
	PSG_CUDA(cudaMalloc(&ctx->d_cell_lo, sizeof(float4) * (ncell + 1)));
	PSG_CUDA(cudaMalloc(&ctx->d_cell_hi, sizeof(float4) * (ncell + 1)));
	k_emit<<<blocks(ncell + 1, 256), 256, 0, st>>>(c, (int)ncell, (uint32_t)nvalid, ctx->d_cell_lo, ctx->d_cell_hi);
	PSG_CHECK_LAUNCH();
	if (ctx->d_wide_lo) cudaFree(ctx->d_wide_lo);
	if (ctx->d_wide_hi) cudaFree(ctx->d_wide_hi);
	ctx->d_wide_lo = ctx->d_wide_hi = nullptr;
	PSG_CUDA(cudaMalloc(&ctx->d_wide_lo, sizeof(float4) * ncell));
	PSG_CUDA(cudaMalloc(&ctx->d_wide_hi, sizeof(float4) * ncell));
	k_emit_wide<<<blocks(ncell, 256), 256, 0, st>>>(c, (int)ncell, ctx->d_wide_lo, ctx->d_wide_hi);
	PSG_CHECK_LAUNCH();
	PSG_CUDA(cudaStreamSynchronize(st));
	ctx->ncell = ncell;
	ctx->nleaf = ncell - (ncell - 1) / 8;
	ctx->nvalid = nvalid;
	ctx->skipped = n - nvalid;
	ctx->depth = nlevels - 1;
	ctx->ppc = ppc;
	ctx->have_tree = 1;
	return PSG_OK;
}

extern "C" int psg_get_tree_info(psg_context *ctx, psg_tree_info *info) {
	if (!ctx || !info) return PSG_E_INVAL;
	if (!ctx->have_tree) return psg_fail(ctx, PSG_E_INVAL, "psg_get_tree_info: no tree");
	info->ncells = ctx->ncell;
	info->nleaves = ctx->nleaf;
	info->skipped = ctx->skipped;
	info->depth = ctx->depth;
	return PSG_OK;
}

extern "C" int psg_get_tree(psg_context *ctx, float *bot, float *top, int32_t *skip,
		int32_t *pstart, int32_t *order) {
	if (!ctx) return PSG_E_INVAL;
	if (!ctx->have_tree) return psg_fail(ctx, PSG_E_INVAL, "psg_get_tree: no tree");
	PSG_CUDA(cudaSetDevice(ctx->device));
	const size_t nc = ctx->ncell;
	std::vector<float4> lo(nc + 1), hi(nc + 1);
	PSG_CUDA(cudaMemcpy(lo.data(), ctx->d_cell_lo, sizeof(float4) * (nc + 1), cudaMemcpyDeviceToHost));
	PSG_CUDA(cudaMemcpy(hi.data(), ctx->d_cell_hi, sizeof(float4) * (nc + 1), cudaMemcpyDeviceToHost));
	for (size_t i = 0; i < nc; i++) {
		if (bot) { bot[3 * i] = lo[i].x; bot[3 * i + 1] = lo[i].y; bot[3 * i + 2] = lo[i].z; }
		if (top) { top[3 * i] = hi[i].x; top[3 * i + 1] = hi[i].y; top[3 * i + 2] = hi[i].z; }
		if (skip) memcpy(&skip[i], &lo[i].w, sizeof(int32_t));
	}
	if (pstart)
		for (size_t i = 0; i <= nc; i++) memcpy(&pstart[i], &hi[i].w, sizeof(int32_t));
	if (order && ctx->nvalid) {
		// leaf order as the caller's particle indices
		std::vector<uint32_t> idx(ctx->nvalid);
		PSG_CUDA(cudaMemcpy(idx.data(), ctx->d_order, sizeof(uint32_t) * ctx->nvalid, cudaMemcpyDeviceToHost));
		for (size_t k = 0; k < ctx->nvalid; k++) order[k] = (int32_t)idx[k];
	}
	return PSG_OK;
}
