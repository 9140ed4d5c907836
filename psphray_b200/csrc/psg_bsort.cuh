// Merge sorts of the rare long lists: by one thread block over an array in
// global memory (a ray with more hits than the shared-memory class sorts
// hold, a particle hit by more rays in one tick than a slot run's shared
// buffer holds), and device-wide (the recombination rays of a tick).
// Tiles of 2 x NT items are bitonic-sorted in shared memory, then merge
// passes of doubling width go between two global buffers; each thread finds
// the start of its share of a merge by a binary search along the merge path
// and merges its share sequentially (on equal items the second run's item
// goes first, in the search and in the merge alike).
#pragma once

namespace {

// Sorts tile[0, 2*NT) in shared memory (padding compares after every real
// item); the caller syncs before, the last step syncs after.
template <int NT, typename Item, typename Less>
__device__ __forceinline__ void tile_bitonic(Item *tile, Less less) {
	constexpr int TS = 2 * NT;
	for (int k = 2; k <= TS; k <<= 1) {
		for (int j = k >> 1; j > 0; j >>= 1) {
			for (int i = threadIdx.x; i < TS; i += NT) {
				const int ixj = i ^ j;
				if (ixj > i) {
					const Item x = tile[i], y = tile[ixj];
					const bool up = (i & k) == 0;
					if (up ? less(y, x) : less(x, y)) {
						tile[i] = y;
						tile[ixj] = x;
					}
				}
			}
			__syncthreads();
		}
	}
}

// Outputs k0 .. k1-1 of the merge of the sorted runs A (la items) and B (lb
// items) into out[k0 .. k1-1].
template <typename Item, typename Less>
__device__ __forceinline__ void merge_slice(const Item *A, int64_t la, const Item *B, int64_t lb, int64_t k0,
		int64_t k1, Item *out, Less less) {
	int64_t lo = max((int64_t)0, k0 - lb), hi = min(k0, la);
	while (lo < hi) {
		const int64_t mid = (lo + hi) >> 1;
		if (less(A[mid], B[k0 - 1 - mid])) lo = mid + 1;
		else hi = mid;
	}
	int64_t i = lo, j = k0 - lo;
	for (int64_t k = k0; k < k1; k++) {
		if (j >= lb || (i < la && less(A[i], B[j]))) out[k] = A[i++];
		else out[k] = B[j++];
	}
}

// One block: a holds the n items on entry; b is scratch of n items. Returns
// the buffer holding the sorted items. Every thread of the block calls it;
// it starts and ends with __syncthreads(). The buffers are read with plain
// loads: they are written inside the same kernel.
template <int NT, typename Item, typename Less>
__device__ Item *block_sort_global(Item *a, Item *b, int64_t n, Item *tile, Item pad, Less less) {
	constexpr int TS = 2 * NT;
	__syncthreads();
	for (int64_t t0 = 0; t0 < n; t0 += TS) {
		const int m = (int)min((int64_t)TS, n - t0);
		for (int i = threadIdx.x; i < TS; i += NT) tile[i] = i < m ? a[t0 + i] : pad;
		__syncthreads();
		tile_bitonic<NT>(tile, less);
		for (int i = threadIdx.x; i < m; i += NT) a[t0 + i] = tile[i];
		__syncthreads();
	}
	for (int64_t w = TS; w < n; w <<= 1) {
		for (int64_t p0 = 0; p0 < n; p0 += 2 * w) {
			const int64_t la = min(w, n - p0);
			const int64_t lb = min(w, n - p0 - la);
			const int64_t L = la + lb;
			const int64_t per = (L + NT - 1) / NT;
			const int64_t k0 = (int64_t)threadIdx.x * per;
			if (k0 < L) merge_slice(a + p0, la, a + p0 + la, lb, k0, min(k0 + per, L), b + p0, less);
		}
		__syncthreads();
		Item *s = a;
		a = b;
		b = s;
	}
	return a;
}

// ---- device-wide: a grid of tiles, then one launch per merge pass ----------
// Tiles of 2 x NT items, NT = 64, 256 or 1024 by the size (a handful of
// recombination rays needs no 1024-thread block).
#define DSORT_PER 8          // outputs per thread in a merge pass (divides every run width)
inline int dsort_nt(size_t n) { return n <= 128 ? 64 : (n <= 512 ? 256 : 1024); }
template <int NT, typename Item, typename Less>
__global__ void __launch_bounds__(NT) k_dsort_tiles(Item *a, size_t n, Item pad, Less less) {
	__shared__ Item tile[2 * NT];
	const size_t t0 = (size_t)blockIdx.x * 2 * NT;
	const int m = (int)min((size_t)2 * NT, n - t0);
	for (int i = threadIdx.x; i < 2 * NT; i += NT) tile[i] = i < m ? a[t0 + i] : pad;
	__syncthreads();
	tile_bitonic<NT>(tile, less);
	for (int i = threadIdx.x; i < m; i += NT) a[t0 + i] = tile[i];
}
template <typename Item, typename Less>
__global__ void __launch_bounds__(256) k_dsort_merge(const Item *__restrict__ a, Item *__restrict__ b, size_t n,
		size_t w, Less less) {
	const size_t k = ((size_t)blockIdx.x * 256 + threadIdx.x) * DSORT_PER;
	if (k >= n) return;
	const size_t p0 = k / (2 * w) * (2 * w);
	const int64_t la = (int64_t)min(w, n - p0);
	const int64_t lb = (int64_t)min(w, n - p0 - (size_t)la);
	merge_slice(a + p0, la, a + p0 + la, lb, (int64_t)(k - p0), (int64_t)min(k - p0 + DSORT_PER, (size_t)(la + lb)),
			b + p0, less);
}
// Number of merge passes after the tiles; the result is in a when even.
inline int dsort_passes(size_t n) {
	int p = 0;
	for (size_t w = 2 * (size_t)dsort_nt(n); w < n; w <<= 1) p++;
	return p;
}
// Issues the sort of a[0, n) (b: scratch of n items) on st; launch sizes
// depend on n alone. The result ends in a or b as dsort_passes(n) says.
template <typename Item, typename Less>
cudaError_t dsort_enqueue(cudaStream_t st, Item *a, Item *b, size_t n, Item pad, Less less) {
	if (n == 0) return cudaSuccess;
	const int nt = dsort_nt(n);
	const unsigned tiles = (unsigned)((n + 2 * nt - 1) / (2 * nt));
	if (nt == 64) k_dsort_tiles<64, Item, Less><<<tiles, 64, 0, st>>>(a, n, pad, less);
	else if (nt == 256) k_dsort_tiles<256, Item, Less><<<tiles, 256, 0, st>>>(a, n, pad, less);
	else k_dsort_tiles<1024, Item, Less><<<tiles, 1024, 0, st>>>(a, n, pad, less);
	for (size_t w = 2 * (size_t)nt; w < n; w <<= 1) {
		k_dsort_merge<Item, Less><<<(unsigned)((n + 256 * DSORT_PER - 1) / (256 * DSORT_PER)), 256, 0, st>>>(a, b, n,
				w, less);
		Item *s = a;
		a = b;
		b = s;
	}
	return cudaGetLastError();
}

}  // namespace
