// Exclusive scans of 64-bit sums over device arrays, used by the traversal
// (hit counts), the tick batches (slots, ray and particle classes) and the
// recombination emission (cumulative weights in FP64, emitter flags); no
// library device-wide scan on the per-step path.
#pragma once

#include <cub/cub.cuh>

#include "psg_internal.cuh"

namespace {

// Exclusive scans of the batch (the slots' (count, count > 0) pairs, the
// traversal's hit counts, the ray and particle classes) in up to three
// passes: tile sums, one block scanning the tile sums, each tile's own scan
// plus its offset. Tiles of 256 threads x 16 items; the element type of the
// input is mapped to the sum's type V (unsigned 64-bit or double) by Op; out
// has n + 1 entries (the total last). The order of the additions is fixed
// by n alone, so a floating-point scan gives the same bits every run.
#define SCAN_T 256
#define SCAN_I 16
struct SlotPair {        // a key's count c: c | (c > 0) << 32 (slots below, active pairs below)
	__device__ __forceinline__ unsigned long long operator()(uint32_t c) const {
		return (unsigned long long)c | ((unsigned long long)(c > 0) << 32);
	}
};
struct Widen {
	template <typename T>
	__device__ __forceinline__ unsigned long long operator()(T c) const { return (unsigned long long)c; }
};
struct AsDouble {
	__device__ __forceinline__ double operator()(double x) const { return x; }
};
template <typename T, typename Op, typename V>
__global__ void __launch_bounds__(SCAN_T) k_scan_tiles(const T *__restrict__ in, size_t n,
		V *__restrict__ tile_sum, Op op) {
	using BR = cub::BlockReduce<V, SCAN_T>;
	__shared__ typename BR::TempStorage tmp;
	const size_t t0 = (size_t)blockIdx.x * SCAN_T * SCAN_I;
	V s = 0;
#pragma unroll
	for (int u = 0; u < SCAN_I; u++) {
		const size_t k = t0 + (size_t)u * SCAN_T + threadIdx.x;
		if (k < n) s += op(in[k]);
	}
	s = BR(tmp).Sum(s);
	if (threadIdx.x == 0) tile_sum[blockIdx.x] = s;
}
// one block: exclusive scan of the tile sums in place; the total after them
template <typename V>
__global__ void __launch_bounds__(1024) k_scan_sums(V *__restrict__ tile_sum, size_t ntile) {
	using BS = cub::BlockScan<V, 1024>;
	__shared__ typename BS::TempStorage tmp;
	__shared__ V carry;
	if (threadIdx.x == 0) carry = 0;
	__syncthreads();
	for (size_t b = 0; b < ntile; b += 1024) {
		const size_t i = b + threadIdx.x;
		const V v = i < ntile ? tile_sum[i] : (V)0;
		V x, agg;
		BS(tmp).ExclusiveSum(v, x, agg);
		if (i < ntile) tile_sum[i] = x + carry;
		__syncthreads();
		if (threadIdx.x == 0) carry += agg;
		__syncthreads();
	}
	if (threadIdx.x == 0) tile_sum[ntile] = carry;
}
// MODE 0: tile_sum holds the tiles' exclusive prefixes (and the total
// after them); MODE 1: tile_sum holds the raw tile sums, and each block sums
// the ones before it itself (few tiles); MODE 2: a single tile, no tile sums.
template <typename T, typename Op, typename V, int MODE>
__global__ void __launch_bounds__(SCAN_T) k_scan_apply(const T *__restrict__ in, size_t n,
		const V *__restrict__ tile_sum, V *__restrict__ out, Op op) {
	using BS = cub::BlockScan<V, SCAN_T>;
	using BR = cub::BlockReduce<V, SCAN_T>;
	__shared__ typename BS::TempStorage tmp;
	__shared__ typename BR::TempStorage rtmp;
	__shared__ V before_s;
	const size_t t0 = (size_t)blockIdx.x * SCAN_T * SCAN_I;
	V before = 0;
	if (MODE == 0) {
		before = tile_sum[blockIdx.x];
	} else if (MODE == 1) {
		V part = 0;
		for (unsigned b = threadIdx.x; b < blockIdx.x; b += SCAN_T) part += tile_sum[b];
		part = BR(rtmp).Sum(part);
		if (threadIdx.x == 0) before_s = part;
		__syncthreads();
		before = before_s;
	}
	// blocked layout: thread i holds items t0 + i*16 .. +15
	V v[SCAN_I];
	V s = 0;
#pragma unroll
	for (int u = 0; u < SCAN_I; u++) {
		const size_t k = t0 + (size_t)threadIdx.x * SCAN_I + u;
		v[u] = k < n ? op(in[k]) : (V)0;
		s += v[u];
	}
	V x;
	BS(tmp).ExclusiveSum(s, x);
	x += before;
#pragma unroll
	for (int u = 0; u < SCAN_I; u++) {
		const size_t k = t0 + (size_t)threadIdx.x * SCAN_I + u;
		if (k < n) out[k] = x;
		x += v[u];
	}
	// the total: the last thread's running sum after its items
	if (blockIdx.x == gridDim.x - 1 && threadIdx.x == SCAN_T - 1) {
		if (MODE == 0) out[n] = tile_sum[gridDim.x];
		else out[n] = x;
	}
}

// Issues the scan on st: out[0..n] (n + 1 entries); tiles: scratch of
// scan_tiles(n) + 1 entries. One launch for a single tile, two up to
// SCAN_FEW tiles (each block sums the tile sums before it), three beyond.
#define SCAN_FEW 256
inline size_t scan_tiles(size_t n) {
	const size_t t = (n + (size_t)SCAN_T * SCAN_I - 1) / ((size_t)SCAN_T * SCAN_I);
	return t ? t : 1;
}
template <typename T, typename Op, typename V>
cudaError_t scan_enqueue(cudaStream_t st, const T *in, size_t n, V *out, V *tiles, Op op) {
	const size_t nt = scan_tiles(n);
	if (nt == 1) {
		k_scan_apply<T, Op, V, 2><<<1, SCAN_T, 0, st>>>(in, n, tiles, out, op);
	} else if (nt <= SCAN_FEW) {
		k_scan_tiles<T, Op, V><<<(unsigned)nt, SCAN_T, 0, st>>>(in, n, tiles, op);
		k_scan_apply<T, Op, V, 1><<<(unsigned)nt, SCAN_T, 0, st>>>(in, n, tiles, out, op);
	} else {
		k_scan_tiles<T, Op, V><<<(unsigned)nt, SCAN_T, 0, st>>>(in, n, tiles, op);
		k_scan_sums<V><<<1, 1024, 0, st>>>(tiles, nt);
		k_scan_apply<T, Op, V, 0><<<(unsigned)nt, SCAN_T, 0, st>>>(in, n, tiles, out, op);
	}
	return cudaGetLastError();
}

}  // namespace
