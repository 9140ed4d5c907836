// The chemistry surrogate inside the ticks (not isothermal): per tick, every
// active particle's step is first predicted by the 5 -> 64 -> 64 -> 2
// network in BF16 on the tensor cores; a cheap residual check accepts the
// prediction or sends the particle to the Dormand-Prince queue.
//
// One CTA of 128 threads takes tiles of 128 particles (one per thread =
// one row of the M = 128 tile). The three layers are tcgen05.mma
// (kind::f16, BF16 operands from shared memory, FP32 accumulators in tensor
// memory): thread 0 issues them, a commit to an mbarrier signals their end,
// every warp reads its 32 rows of the accumulator with tcgen05.ld, adds the
// bias, applies SiLU and writes the BF16 activations back as the next
// layer's A operand. Weights sit in shared memory for the kernel's life.
//
// Operands use the no-swizzle K-major layout: 8 rows x 16 bytes form a core
// matrix (128 contiguous bytes); element (row r, k) of a matrix with R rows
// sits at byte ((k/8)*(R/8) + r/8)*128 + (r%8)*16 + (k%8)*2, so the stride
// between 8-row groups (SBO) is 128 B and between 8-column chunks (LBO) is
// R*16 B. One MMA consumes K = 16, i.e. two chunks.
//
// The residual check is the trapezoid rule of the step's ODE (solve.c:
// 76-141): r = x1 - x0 - (f(x0) + f(x1))/2 over the normalised step, for
// x = (lambdaH, ie); the prediction stands if |r_lambda| <= tol *
// max(min(lambda, 1 - lambda), 1e-6) and |r_ie| <= tol * ie.
#include <cuda_bf16.h>
#include <string.h>

#include <vector>

#include "psg_internal.cuh"
#include "psg_surrogate.cuh"

namespace {

constexpr int M = 128, H = 64, K1 = 16, N3 = 16;
// byte offsets inside the weight blob (global) and in shared memory
constexpr int W1_BYTES = H * K1 * 2, W2_BYTES = H * H * 2, W3_BYTES = N3 * H * 2;
constexpr int OFF_W1 = 0, OFF_W2 = OFF_W1 + W1_BYTES, OFF_W3 = OFF_W2 + W2_BYTES;
constexpr int OFF_B1 = OFF_W3 + W3_BYTES, OFF_B2 = OFF_B1 + H * 4, OFF_B3 = OFF_B2 + H * 4;
constexpr int BLOB_BYTES = OFF_B3 + 16 * 4;     // b3[2], ymu[2], ystd[2], pad
constexpr int A_BYTES = M * H * 2;
constexpr int SMEM_BYTES = A_BYTES + BLOB_BYTES + 64;
static_assert(BLOB_BYTES % 16 == 0, "blob");

__host__ __device__ constexpr int blocked(int rows, int r, int k) {
	return ((k / 8) * (rows / 8) + r / 8) * 128 + (r % 8) * 16 + (k % 8) * 2;
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
	return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
			((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// kind::f16 instruction descriptor: BF16 A and B, FP32 D, both K-major
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n) {
	return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
	asm volatile(
			"{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
			"tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
			"l"(a), "l"(b), "r"(idesc), "r"(acc)
			: "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
	asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
			: "memory");
}

// bounded wait on an mbarrier phase; false if it never completed
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t phase) {
	for (int i = 0; i < (1 << 22); i++) {
		uint32_t done;
		asm volatile(
				"{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
				"selp.u32 %0, 1, 0, p;\n\t}\n"
				: "=r"(done)
				: "r"(mbar), "r"(phase)
				: "memory");
		if (done) return true;
	}
	return false;
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16]) {
	uint32_t r[16];
	asm volatile(
			"tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
			: "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
			"=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
			: "r"(taddr));
	asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
	for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
	const __nv_bfloat16 x = __float2bfloat16_rn(a), y = __float2bfloat16_rn(b);
	return (uint32_t)__bfloat16_as_ushort(x) | ((uint32_t)__bfloat16_as_ushort(y) << 16);
}

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }

// Bias + SiLU of this thread's 64 accumulators (row `row`), written to A as
// BF16 in the blocked layout.
__device__ __forceinline__ void epilogue_hidden(uint32_t tmem_row, const float *b, char *A, int row) {
#pragma unroll
	for (int q = 0; q < 4; q++) {
		float v[16];
		tmem_ld16(tmem_row + q * 16, v);
#pragma unroll
		for (int h = 0; h < 2; h++) {
			const int c = q * 2 + h;     // chunk of 8 columns
			uint4 w;
			w.x = pack_bf16(silu(v[h * 8 + 0] + b[c * 8 + 0]), silu(v[h * 8 + 1] + b[c * 8 + 1]));
			w.y = pack_bf16(silu(v[h * 8 + 2] + b[c * 8 + 2]), silu(v[h * 8 + 3] + b[c * 8 + 3]));
			w.z = pack_bf16(silu(v[h * 8 + 4] + b[c * 8 + 4]), silu(v[h * 8 + 5] + b[c * 8 + 5]));
			w.w = pack_bf16(silu(v[h * 8 + 6] + b[c * 8 + 6]), silu(v[h * 8 + 7] + b[c * 8 + 7]));
			*(uint4 *)(A + blocked(M, row, c * 8)) = w;
		}
	}
}

// RAW: rows of raw inputs (8 floats, 5 used) in, the de-normalised outputs
// (2 floats per row) out -- the network alone, for checks and evaluation.
struct RawIO {
	const float *x;
	float *y;
	int n;
};

template <bool RAW>
__global__ void __launch_bounds__(128, 4) k_surrogate(int t, const int32_t *__restrict__ tick_act,
		const uint32_t *__restrict__ act_ipar, const double *__restrict__ act_g, const double *__restrict__ act_heat,
		double *__restrict__ lambdaH, float *__restrict__ ie, int64_t *__restrict__ lasthit,
		const float *__restrict__ rho, const float *__restrict__ yeMET, PhysParams P,
		const PsgBatchDev *__restrict__ B, const char *__restrict__ blob, float tol, uint32_t *__restrict__ rej,
		unsigned *__restrict__ nrej, unsigned long long *__restrict__ nacc, uint32_t *__restrict__ status, RawIO io) {
	extern __shared__ __align__(1024) char smem[];
	char *A = smem;
	char *Wsm = smem + A_BYTES;
	uint64_t *mbar = (uint64_t *)(Wsm + BLOB_BYTES);
	uint32_t *tmem_slot = (uint32_t *)(Wsm + BLOB_BYTES + 16);
	const int tid = threadIdx.x, warp = tid >> 5;
	const int lo = RAW ? 0 : tick_act[t], hi = RAW ? io.n : tick_act[t + 1];
	const int64_t tick = RAW ? 0 : B->tick0 + t;
	const double tick_time = RAW ? 0.0 : B->tick_time;
	const int ntile = (hi - lo + M - 1) / M;
	if ((int)blockIdx.x >= ntile) return;

	for (int i = tid * 16; i < BLOB_BYTES; i += 128 * 16) *(uint4 *)(Wsm + i) = *(const uint4 *)(blob + i);
	const uint32_t mbar_a = (uint32_t)__cvta_generic_to_shared(mbar);
	if (tid == 0) {
		asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar_a) : "memory");
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	}
	if (warp == 0) {
		asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 64;" ::"r"(
				(uint32_t)__cvta_generic_to_shared(tmem_slot))
				: "memory");
		asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
	}
	fence_before();
	__syncthreads();
	fence_after();
	const uint32_t tmem = *tmem_slot;
	const uint32_t tmem_row = tmem + ((uint32_t)(warp * 32) << 16);
	const float *b1 = (const float *)(Wsm + OFF_B1), *b2 = (const float *)(Wsm + OFF_B2);
	const float *b3 = (const float *)(Wsm + OFF_B3);
	const uint32_t a_addr = (uint32_t)__cvta_generic_to_shared(A);
	const uint32_t w_addr = (uint32_t)__cvta_generic_to_shared(Wsm);
	uint32_t phase = 0;
	bool ok = true;
	uint32_t st = 0;

	for (int tile = blockIdx.x; tile < ntile && ok; tile += gridDim.x) {
		const int a = lo + tile * M + tid;
		const bool mine = a < hi;
		// this thread's particle and its inputs (row tid of the first A)
		uint32_t p = 0;
		double lam0 = 0.0, ie0 = 1.0;
		RhsCtx cx{};
		float f[PSG_SURR_NFEAT] = {0.f, 0.f, 0.f, 0.f, 0.f};
		if (RAW && mine) {
			for (int k = 0; k < PSG_SURR_NFEAT; k++) f[k] = io.x[(size_t)a * 8 + k];
		} else if (mine) {
			p = act_ipar[a];
			const double time = rn_dmul((double)(tick - lasthit[p]), tick_time);
			lam0 = lambdaH[p];
			ie0 = (double)ie[p];
			const double T = ieye2T(P, ie0, rn_dadd(rn_dsub(1.0, lam0), P.he_e));
			cx = make_rhs_ctx(P, (double)yeMET[p], act_g[a], act_heat[a], time, rn_dmul(P.H_PER_MASS, (double)rho[p]), T);
			surr_features(cx, lam0, ie0, f);
		}
		{
			uint4 w0, w1;
			w0.x = pack_bf16(f[0], f[1]);
			w0.y = pack_bf16(f[2], f[3]);
			w0.z = pack_bf16(f[4], 0.f);
			w0.w = 0u;
			w1.x = w1.y = w1.z = w1.w = 0u;
			*(uint4 *)(A + blocked(M, tid, 0)) = w0;
			*(uint4 *)(A + blocked(M, tid, 8)) = w1;
		}
		fence_async_smem();
		fence_before();
		__syncthreads();
		fence_after();
		// layer 1: D[128 x 64] = A[128 x 16] W1^T
		if (tid == 0) {
			mma_bf16(tmem, smem_desc(a_addr, M * 16, 128), smem_desc(w_addr + OFF_W1, H * 16, 128), idesc_bf16(M, H), 0);
			mma_commit(mbar_a);
		}
		ok = mbar_wait(mbar_a, phase);
		phase ^= 1;
		fence_after();
		if (ok) epilogue_hidden(tmem_row, b1, A, tid);
		fence_async_smem();
		fence_before();
		__syncthreads();
		fence_after();
		if (!__syncthreads_and(ok)) { ok = false; break; }
		// layer 2: D[128 x 64] = A[128 x 64] W2^T, four K = 16 steps
		if (tid == 0) {
#pragma unroll
			for (int j = 0; j < 4; j++)
				mma_bf16(tmem, smem_desc(a_addr + j * 2 * M * 16, M * 16, 128),
						smem_desc(w_addr + OFF_W2 + j * 2 * H * 16, H * 16, 128), idesc_bf16(M, H), j > 0);
			mma_commit(mbar_a);
		}
		ok = mbar_wait(mbar_a, phase);
		phase ^= 1;
		fence_after();
		if (ok) epilogue_hidden(tmem_row, b2, A, tid);
		fence_async_smem();
		fence_before();
		__syncthreads();
		fence_after();
		if (!__syncthreads_and(ok)) { ok = false; break; }
		// layer 3: D[128 x 16] = A[128 x 64] W3^T (2 of the 16 outputs used)
		if (tid == 0) {
#pragma unroll
			for (int j = 0; j < 4; j++)
				mma_bf16(tmem, smem_desc(a_addr + j * 2 * M * 16, M * 16, 128),
						smem_desc(w_addr + OFF_W3 + j * 2 * N3 * 16, N3 * 16, 128), idesc_bf16(M, N3), j > 0);
			mma_commit(mbar_a);
		}
		ok = mbar_wait(mbar_a, phase);
		phase ^= 1;
		fence_after();
		float out[16];
		if (ok) tmem_ld16(tmem_row, out);
		fence_before();
		__syncthreads();
		fence_after();
		if (!__syncthreads_and(ok)) { ok = false; break; }
		if (!mine) continue;
		// prediction -> state, then the trapezoid residual
		const double y0 = (double)(out[0] + b3[0]) * (double)b3[4] + (double)b3[2];
		const double y1 = (double)(out[1] + b3[1]) * (double)b3[5] + (double)b3[3];
		if (RAW) {
			io.y[(size_t)a * 2] = (float)y0;
			io.y[(size_t)a * 2 + 1] = (float)y1;
			continue;
		}
		const double lam1 = surr_unlogit((double)f[2] + y0);
		const double T1 = exp10((double)f[1] + y1);
		const double ie1 = Tye2ie(P, T1, rn_dadd(rn_dsub(1.0, lam1), P.he_e));
		bool accept = isfinite(lam1) && isfinite(ie1) && ie1 > 0.0 && lam1 >= 0.0 && lam1 <= 1.0;
		if (accept) {
			const double x0[2] = {lam0, ie0}, x1[2] = {lam1, ie1};
			double f0[2], f1[2];
			rhs(P, cx, x0, f0);
			rhs(P, cx, x1, f1);
			const double r0 = lam1 - lam0 - 0.5 * (f0[0] + f1[0]);
			const double r1 = ie1 - ie0 - 0.5 * (f0[1] + f1[1]);
			accept = fabs(r0) <= tol * fmax(fmin(lam1, 1.0 - lam1), 1e-6) && fabs(r1) <= tol * ie1;
		}
		if (accept) {
			lambdaH[p] = lam1;
			ie[p] = (float)ie1;
			lasthit[p] = tick;
		}
		if (!accept) rej[atomicAdd(nrej, 1u)] = (uint32_t)a;
		else atomicAdd(nacc, 1ull);
	}
	if (!ok) st |= PSG_ST_SURR;
	fence_before();
	__syncthreads();
	fence_after();
	if (warp == 0)
		asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 64;" ::"r"(tmem) : "memory");
	if (st && tid == 0) atomicOr(status, st);
}

}  // namespace

// Weight blob in the kernel's shared-memory image: BF16 weights in the
// blocked layout (input normalisation folded into W1, b1), FP32 biases,
// output de-normalisation.
int psg_surrogate_blob(const float *params, const float *x_mu, const float *x_sd, const float *y_mu,
		const float *y_sd, std::vector<char> &blob) {
	blob.assign(BLOB_BYTES, 0);
	const float *W1 = params, *b1 = params + 64 * PSG_MLP_NIN, *W2 = b1 + 64, *b2 = W2 + 64 * 64, *W3 = b2 + 64;
	const float *b3 = W3 + 2 * 64;
	auto put = [&](int off, float v) {
		const __nv_bfloat16 h = __float2bfloat16_rn(v);
		const unsigned short u = __bfloat16_as_ushort(h);
		memcpy(&blob[off], &u, 2);
	};
	float *fb1 = (float *)&blob[OFF_B1], *fb2 = (float *)&blob[OFF_B2], *fb3 = (float *)&blob[OFF_B3];
	for (int j = 0; j < 64; j++) {
		double bias = b1[j];
		for (int k = 0; k < PSG_SURR_NFEAT; k++) {
			const double w = (double)W1[j * PSG_MLP_NIN + k] / (double)x_sd[k];
			put(OFF_W1 + blocked(64, j, k), (float)w);
			bias -= w * (double)x_mu[k];
		}
		fb1[j] = (float)bias;
		for (int k = 0; k < 64; k++) put(OFF_W2 + blocked(64, j, k), W2[j * 64 + k]);
		fb2[j] = b2[j];
	}
	for (int o = 0; o < 2; o++)
		for (int k = 0; k < 64; k++) put(OFF_W3 + blocked(N3, o, k), W3[o * 64 + k]);
	fb3[0] = b3[0];
	fb3[1] = b3[1];
	fb3[2] = y_mu[0];
	fb3[3] = y_mu[1];
	fb3[4] = y_sd[0];
	fb3[5] = y_sd[1];
	return PSG_OK;
}

extern "C" int psg_set_surrogate(psg_context *ctx, const float *params, const float *x_mu, const float *x_sd,
		const float *y_mu, const float *y_sd, float tol) {
	if (!ctx) return PSG_E_INVAL;
	PSG_CUDA(cudaSetDevice(ctx->device));
	if (!params) {
		ctx->surr_on = 0;
		return PSG_OK;
	}
	if (!x_mu || !x_sd || !y_mu || !y_sd || !(tol > 0.0f))
		return psg_fail(ctx, PSG_E_INVAL, "psg_set_surrogate: normalisation and a positive tolerance are required");
	for (int k = 0; k < PSG_SURR_NFEAT; k++)
		if (!(x_sd[k] > 0.0f)) return psg_fail(ctx, PSG_E_INVAL, "psg_set_surrogate: input scale %d not positive", k);
	std::vector<char> blob;
	psg_surrogate_blob(params, x_mu, x_sd, y_mu, y_sd, blob);
	if (!ctx->d_surr) PSG_CUDA(cudaMalloc(&ctx->d_surr, BLOB_BYTES));
	PSG_CUDA(cudaMemcpyAsync(ctx->d_surr, blob.data(), BLOB_BYTES, cudaMemcpyHostToDevice, ctx->stream));
	PSG_CUDA(cudaStreamSynchronize(ctx->stream));
	ctx->surr_tol = tol;
	ctx->surr_on = 1;
	return PSG_OK;
}

// Runs the surrogate over tick t's active particles; rejected ones are
// listed in rej (count in *nrej, on the device).
int psg_surrogate_prepare(psg_context *ctx) {
	PSG_CUDA(cudaFuncSetAttribute(k_surrogate<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES));
	return PSG_OK;
}

int psg_surrogate_tick(psg_context *ctx, int t, const int32_t *tick_act, const uint32_t *act_ipar,
		const double *act_g, const double *act_heat, const PhysParams &P, const PsgBatchDev *B, uint32_t *rej,
		unsigned *nrej) {
	static_assert(SMEM_BYTES < 200 * 1024, "smem");
	cudaStream_t st = ctx->stream;
	// a persistent grid: the tick's particle count is read on the device
	const unsigned grid = (unsigned)(ctx->sms * 4);
	k_surrogate<false><<<grid, 128, SMEM_BYTES, st>>>(t, tick_act, act_ipar, act_g, act_heat, ctx->d_lambdaH,
			ctx->d_ie, ctx->d_lasthit, ctx->d_rho, ctx->d_yeMET, P, B, (const char *)ctx->d_surr,
			ctx->surr_tol, rej, nrej, ctx->d_counters + 8, ctx->d_status, RawIO{nullptr, nullptr, 0});
	PSG_CHECK_LAUNCH();
	return PSG_OK;
}

extern "C" int psg_surrogate_forward(psg_context *ctx, const float *d_x, size_t n, float *d_y) {
	if (!ctx) return PSG_E_INVAL;
	if (!ctx->surr_on || !ctx->d_surr) return psg_fail(ctx, PSG_E_INVAL, "psg_surrogate_forward: no surrogate set");
	if (!d_x || !d_y || n >= (size_t)INT32_MAX) return psg_fail(ctx, PSG_E_INVAL, "psg_surrogate_forward: bad argument");
	if (n == 0) return PSG_OK;
	PSG_CUDA(cudaSetDevice(ctx->device));
	int sms = 148;
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
	PSG_CUDA(cudaFuncSetAttribute(k_surrogate<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES));
	const int ntile = (int)((n + M - 1) / M);
	const unsigned grid = (unsigned)std::min(ntile, sms * 4);
	PhysParams P{};
	PSG_CUDA(cudaMemsetAsync(ctx->d_status, 0, sizeof(uint32_t), ctx->stream));
	k_surrogate<true><<<grid, 128, SMEM_BYTES, ctx->stream>>>(0, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
			nullptr, nullptr, nullptr, P, nullptr, (const char *)ctx->d_surr, ctx->surr_tol, nullptr, nullptr, nullptr,
			ctx->d_status, RawIO{d_x, d_y, (int)n});
	PSG_CHECK_LAUNCH();
	uint32_t st = 0;
	PSG_CUDA(cudaMemcpyAsync(&st, ctx->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
	PSG_CUDA(cudaStreamSynchronize(ctx->stream));
	if (st) return psg_fail(ctx, PSG_E_DEVICE, "psg_surrogate_forward: device status 0x%x", st);
	return PSG_OK;
}
