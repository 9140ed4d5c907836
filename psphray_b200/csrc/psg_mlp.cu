// The chemistry surrogate's network, trained on the device: a 6 -> 64 -> 64
// -> 2 multilayer perceptron with SiLU activations, in FP32 (training) on
// the CUDA cores. Inference inside the ticks runs the same network in BF16
// on the tensor cores (psg_surrogate.cu).
//
// Parameters are one flat FP32 array (PSG_MLP_NPARAM floats):
//   W1[64][8] (inputs padded to 8), b1[64], W2[64][64], b2[64], W3[2][64], b3[2]
// Samples are rows of PSG_MLP_NIN (8) normalised inputs and 2 normalised
// targets. The loss is the mean over samples of the summed squared error.
//
// Gradients are deterministic: every block sums its samples' gradients in a
// fixed order into its own partial, and a second kernel adds the partials
// in block order.
#include <math.h>

#include "psg_internal.cuh"

namespace {

constexpr int NIN = PSG_MLP_NIN, H = 64, NOUT = 2;
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + H * NIN, OFF_W2 = OFF_B1 + H, OFF_B2 = OFF_W2 + H * H,
		OFF_W3 = OFF_B2 + H, OFF_B3 = OFF_W3 + NOUT * H, NPARAM = OFF_B3 + NOUT;
static_assert(NPARAM == PSG_MLP_NPARAM, "parameter layout");
constexpr int BS = 64;          // samples per block iteration
constexpr int TPB = 256;

__device__ __forceinline__ float sigm(float z) { return 1.0f / (1.0f + expf(-z)); }

struct MlpSmem {
	float p[NPARAM];
	float g[NPARAM];
	float x[BS][NIN];
	float t[BS][NOUT];
	float z1[BS][H], h1[BS][H], z2[BS][H], h2[BS][H];
	float y[BS][NOUT];
	float loss;
};

// Forward pass of BS samples already in sm.x (rows >= nb are zero).
__device__ void forward(MlpSmem &sm) {
	const float *W1 = sm.p + OFF_W1, *b1 = sm.p + OFF_B1, *W2 = sm.p + OFF_W2, *b2 = sm.p + OFF_B2;
	const float *W3 = sm.p + OFF_W3, *b3 = sm.p + OFF_B3;
	for (int i = threadIdx.x; i < BS * H; i += TPB) {
		const int s = i / H, j = i % H;
		float z = b1[j];
		for (int k = 0; k < NIN; k++) z = fmaf(W1[j * NIN + k], sm.x[s][k], z);
		sm.z1[s][j] = z;
		sm.h1[s][j] = z * sigm(z);
	}
	__syncthreads();
	for (int i = threadIdx.x; i < BS * H; i += TPB) {
		const int s = i / H, j = i % H;
		float z = b2[j];
		for (int k = 0; k < H; k++) z = fmaf(W2[j * H + k], sm.h1[s][k], z);
		sm.z2[s][j] = z;
		sm.h2[s][j] = z * sigm(z);
	}
	__syncthreads();
	for (int i = threadIdx.x; i < BS * NOUT; i += TPB) {
		const int s = i / NOUT, o = i % NOUT;
		float y = b3[o];
		for (int k = 0; k < H; k++) y = fmaf(W3[o * H + k], sm.h2[s][k], y);
		sm.y[s][o] = y;
	}
	__syncthreads();
}

__device__ void load_rows(MlpSmem &sm, const float *X, const float *T, size_t s0, int nb) {
	for (int i = threadIdx.x; i < BS * NIN; i += TPB) {
		const int s = i / NIN, k = i % NIN;
		sm.x[s][k] = s < nb ? X[(s0 + s) * NIN + k] : 0.0f;
	}
	if (T)
		for (int i = threadIdx.x; i < BS * NOUT; i += TPB) {
			const int s = i / NOUT, o = i % NOUT;
			sm.t[s][o] = s < nb ? T[(s0 + s) * NOUT + o] : 0.0f;
		}
	__syncthreads();
}

__global__ void __launch_bounds__(TPB) k_mlp_forward(const float *__restrict__ params, const float *__restrict__ X,
		size_t n, float *__restrict__ Y) {
	extern __shared__ __align__(16) char smem_raw[];
	MlpSmem &sm = *reinterpret_cast<MlpSmem *>(smem_raw);
	for (int i = threadIdx.x; i < NPARAM; i += TPB) sm.p[i] = params[i];
	__syncthreads();
	for (size_t s0 = (size_t)blockIdx.x * BS; s0 < n; s0 += (size_t)gridDim.x * BS) {
		const int nb = (int)min((size_t)BS, n - s0);
		load_rows(sm, X, nullptr, s0, nb);
		forward(sm);
		for (int i = threadIdx.x; i < nb * NOUT; i += TPB) Y[s0 * NOUT + i] = sm.y[i / NOUT][i % NOUT];
		__syncthreads();
	}
}

// Loss and gradient partial of each block (partials[block][NPARAM + 1], the
// last entry the block's summed squared error).
__global__ void __launch_bounds__(TPB) k_mlp_grad(const float *__restrict__ params, const float *__restrict__ X,
		const float *__restrict__ T, size_t n, float scale, float *__restrict__ partials) {
	extern __shared__ __align__(16) char smem_raw[];
	MlpSmem &sm = *reinterpret_cast<MlpSmem *>(smem_raw);
	for (int i = threadIdx.x; i < NPARAM; i += TPB) {
		sm.p[i] = params[i];
		sm.g[i] = 0.0f;
	}
	if (threadIdx.x == 0) sm.loss = 0.0f;
	__syncthreads();
	const float *W2 = sm.p + OFF_W2, *W3 = sm.p + OFF_W3;
	float *gW1 = sm.g + OFF_W1, *gb1 = sm.g + OFF_B1, *gW2 = sm.g + OFF_W2, *gb2 = sm.g + OFF_B2;
	float *gW3 = sm.g + OFF_W3, *gb3 = sm.g + OFF_B3;
	for (size_t s0 = (size_t)blockIdx.x * BS; s0 < n; s0 += (size_t)gridDim.x * BS) {
		const int nb = (int)min((size_t)BS, n - s0);
		load_rows(sm, X, T, s0, nb);
		forward(sm);
		// dL/dy = 2 (y - t) * scale, zero for padding rows; y reused for it
		if (threadIdx.x == 0) {
			float l = 0.0f;
			for (int s = 0; s < nb; s++)
				for (int o = 0; o < NOUT; o++) {
					const float d = sm.y[s][o] - sm.t[s][o];
					l = fmaf(d, d, l);
				}
			sm.loss += l;
		}
		__syncthreads();
		for (int i = threadIdx.x; i < BS * NOUT; i += TPB) {
			const int s = i / NOUT, o = i % NOUT;
			sm.y[s][o] = s < nb ? 2.0f * (sm.y[s][o] - sm.t[s][o]) * scale : 0.0f;
		}
		__syncthreads();
		// layer 3
		for (int i = threadIdx.x; i < NOUT * H; i += TPB) {
			const int o = i / H, k = i % H;
			float a = 0.0f;
			for (int s = 0; s < nb; s++) a = fmaf(sm.y[s][o], sm.h2[s][k], a);
			gW3[o * H + k] += a;
		}
		if (threadIdx.x < NOUT) {
			float a = 0.0f;
			for (int s = 0; s < nb; s++) a += sm.y[s][threadIdx.x];
			gb3[threadIdx.x] += a;
		}
		__syncthreads();
		// dZ2 into h2
		for (int i = threadIdx.x; i < BS * H; i += TPB) {
			const int s = i / H, k = i % H;
			float d = 0.0f;
			for (int o = 0; o < NOUT; o++) d = fmaf(sm.y[s][o], W3[o * H + k], d);
			const float z = sm.z2[s][k], sg = sigm(z);
			sm.h2[s][k] = d * sg * (1.0f + z * (1.0f - sg));
		}
		__syncthreads();
		// layer 2
		for (int i = threadIdx.x; i < H * H; i += TPB) {
			const int j = i / H, k = i % H;
			float a = 0.0f;
			for (int s = 0; s < nb; s++) a = fmaf(sm.h2[s][j], sm.h1[s][k], a);
			gW2[j * H + k] += a;
		}
		if (threadIdx.x < H) {
			float a = 0.0f;
			for (int s = 0; s < nb; s++) a += sm.h2[s][threadIdx.x];
			gb2[threadIdx.x] += a;
		}
		__syncthreads();
		// dZ1 into h1
		for (int i = threadIdx.x; i < BS * H; i += TPB) {
			const int s = i / H, k = i % H;
			float d = 0.0f;
			for (int j = 0; j < H; j++) d = fmaf(sm.h2[s][j], W2[j * H + k], d);
			const float z = sm.z1[s][k], sg = sigm(z);
			sm.h1[s][k] = d * sg * (1.0f + z * (1.0f - sg));
		}
		__syncthreads();
		// layer 1
		for (int i = threadIdx.x; i < H * NIN; i += TPB) {
			const int j = i / NIN, k = i % NIN;
			float a = 0.0f;
			for (int s = 0; s < nb; s++) a = fmaf(sm.h1[s][j], sm.x[s][k], a);
			gW1[j * NIN + k] += a;
		}
		if (threadIdx.x < H) {
			float a = 0.0f;
			for (int s = 0; s < nb; s++) a += sm.h1[s][threadIdx.x];
			gb1[threadIdx.x] += a;
		}
		__syncthreads();
	}
	float *out = partials + (size_t)blockIdx.x * (NPARAM + 1);
	for (int i = threadIdx.x; i < NPARAM; i += TPB) out[i] = sm.g[i];
	if (threadIdx.x == 0) out[NPARAM] = sm.loss;
}

__global__ void k_mlp_sum_partials(const float *__restrict__ partials, int nblocks, float *__restrict__ grad) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i > NPARAM) return;
	float a = 0.0f;
	for (int b = 0; b < nblocks; b++) a += partials[(size_t)b * (NPARAM + 1) + i];
	grad[i] = a;
}

__global__ void k_mlp_adam(float *__restrict__ params, const float *__restrict__ grad, float *__restrict__ m,
		float *__restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= NPARAM) return;
	const float g = grad[i];
	const float mi = b1 * m[i] + (1.0f - b1) * g;
	const float vi = b2 * v[i] + (1.0f - b2) * g * g;
	m[i] = mi;
	v[i] = vi;
	params[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

int mlp_smem(psg_context *ctx, const void *kern) {
	const int smem = (int)sizeof(MlpSmem);
	const cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
	if (e != cudaSuccess) return psg_cuda_fail(ctx, e, "cudaFuncSetAttribute(mlp)", __FILE__, __LINE__);
	return PSG_OK;
}

}  // namespace

extern "C" int psg_mlp_forward(psg_context *ctx, const float *d_params, const float *d_x, size_t n, float *d_y) {
	if (!ctx) return PSG_E_INVAL;
	if (!d_params || !d_x || !d_y) return psg_fail(ctx, PSG_E_INVAL, "psg_mlp_forward: null pointer");
	if (n == 0) return PSG_OK;
	PSG_CUDA(cudaSetDevice(ctx->device));
	int rc = mlp_smem(ctx, (const void *)k_mlp_forward);
	if (rc) return rc;
	const unsigned grid = (unsigned)std::min<size_t>((n + BS - 1) / BS, 148 * 4);
	k_mlp_forward<<<grid, TPB, sizeof(MlpSmem), ctx->stream>>>(d_params, d_x, n, d_y);
	PSG_CHECK_LAUNCH();
	return PSG_OK;
}

extern "C" int psg_mlp_grad(psg_context *ctx, const float *d_params, const float *d_x, const float *d_t, size_t n,
		float *d_grad, float *d_loss) {
	if (!ctx) return PSG_E_INVAL;
	if (!d_params || !d_x || !d_t || !d_grad || n == 0) return psg_fail(ctx, PSG_E_INVAL, "psg_mlp_grad: bad argument");
	PSG_CUDA(cudaSetDevice(ctx->device));
	int rc = mlp_smem(ctx, (const void *)k_mlp_grad);
	if (rc) return rc;
	const int nblocks = (int)std::min<size_t>((n + BS - 1) / BS, 148 * 2);
	float *partials = (float *)psg_scratch(ctx, S_MLP, sizeof(float) * (size_t)nblocks * (NPARAM + 1));
	if (!partials) return PSG_E_NOMEM;
	k_mlp_grad<<<nblocks, TPB, sizeof(MlpSmem), ctx->stream>>>(d_params, d_x, d_t, n, 1.0f / (float)n, partials);
	PSG_CHECK_LAUNCH();
	// grad[NPARAM] receives the summed squared error
	float *gl = d_grad;
	k_mlp_sum_partials<<<(NPARAM + 256) / 256, 256, 0, ctx->stream>>>(partials, nblocks, gl);
	PSG_CHECK_LAUNCH();
	if (d_loss) PSG_CUDA(cudaMemcpyAsync(d_loss, gl + NPARAM, sizeof(float), cudaMemcpyDeviceToDevice, ctx->stream));
	return PSG_OK;
}

extern "C" int psg_mlp_adam(psg_context *ctx, float *d_params, const float *d_grad, float *d_m, float *d_v,
		float lr, float beta1, float beta2, float eps, int step) {
	if (!ctx) return PSG_E_INVAL;
	if (!d_params || !d_grad || !d_m || !d_v || step < 1) return psg_fail(ctx, PSG_E_INVAL, "psg_mlp_adam: bad argument");
	PSG_CUDA(cudaSetDevice(ctx->device));
	const float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
	k_mlp_adam<<<(NPARAM + 255) / 256, 256, 0, ctx->stream>>>(d_params, d_grad, d_m, d_v, lr, beta1, beta2, eps, c1, c2);
	PSG_CHECK_LAUNCH();
	return PSG_OK;
}
