// Counter-based random numbers shared by the emission kernels (source rays,
// psg_emit.cu; recombination rays, psg_recomb.cu): Philox4x32-10 (Salmon,
// Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3",
// SC'11), counter = (draw index within the tick, tick low word, tick high
// word, stream), key = the 64-bit seed. Streams: 0 source choice, 1 point
// source direction, 2 spectrum energy, 3 plane source position, 4 HII
// recombination emitter, 5 recombination direction, 6 recombination
// energy, 7 and 8 HeII and HeIII recombination emitters.
#pragma once

#include <stdint.h>

// Philox4x32-10: 10 rounds of two 32x32->64 multiplications, the key
// bumped by the Weyl constants between rounds.
static __device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
	for (int r = 0; r < 10; r++) {
		if (r) {
			k0 += 0x9E3779B9u;
			k1 += 0xBB67AE85u;
		}
		const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
		const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
		const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0;
		const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
		c[1] = (uint32_t)p1;
		c[3] = (uint32_t)p0;
		c[0] = n0;
		c[2] = n2;
	}
}

static __device__ __forceinline__ double u01(uint32_t hi, uint32_t lo) {
	return (double)((((uint64_t)hi << 32) | lo) >> 11) * 0x1.0p-53;
}

static __device__ __forceinline__ void draw(uint32_t out[4], uint32_t ray, int64_t tick, uint32_t stream, uint64_t seed) {
	out[0] = ray;
	out[1] = (uint32_t)(uint64_t)tick;
	out[2] = (uint32_t)((uint64_t)tick >> 32);
	out[3] = stream;
	philox4x32_10(out, (uint32_t)seed, (uint32_t)(seed >> 32));
}

// first i in [lo, hi) with cdf[i] > target, or hi
static __device__ __forceinline__ int upper_index(const double *cdf, int lo, int hi, double target) {
	while (lo < hi) {
		const int mid = (lo + hi) >> 1;
		if (cdf[mid] > target) hi = mid;
		else lo = mid + 1;
	}
	return lo;
}

