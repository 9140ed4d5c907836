// Context lifetime, error reporting, physics tables and particle upload.
#include <math.h>
#include <stdarg.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include <mutex>

#include "psg_internal.cuh"

int psg_fail(psg_context *ctx, int code, const char *fmt, ...) {
	if (ctx) {
		va_list ap;
		va_start(ap, fmt);
		vsnprintf(ctx->err, sizeof(ctx->err), fmt, ap);
		va_end(ap);
	}
	return code;
}

int psg_cuda_fail(psg_context *ctx, cudaError_t e, const char *what, const char *file, int line) {
	const int code = (e == cudaErrorMemoryAllocation) ? PSG_E_NOMEM : PSG_E_CUDA;
	return psg_fail(ctx, code, "%s: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
}

void *psg_scratch(psg_context *ctx, int slot, size_t bytes) {
	if (slot < 0 || slot >= S_NSLOTS) return nullptr;
	psg_buf &b = ctx->scratch[slot];
	if (b.bytes >= bytes && b.p) return b.p;
	if (b.p) cudaFree(b.p);
	b.p = nullptr;
	b.bytes = 0;
	size_t want = bytes + bytes / 4 + 256;
	if (cudaMalloc(&b.p, want) != cudaSuccess) {
		cudaGetLastError();
		b.p = nullptr;
		psg_fail(ctx, PSG_E_NOMEM, "device allocation of %zu bytes failed (scratch %d)", want, slot);
		return nullptr;
	}
	b.bytes = want;
	return b.p;
}

extern "C" int psg_create(psg_context **out, int device) {
	if (!out) return PSG_E_INVAL;
	*out = nullptr;
	int ndev = 0;
	cudaError_t e = cudaGetDeviceCount(&ndev);
	if (e != cudaSuccess || ndev == 0) {
		cudaGetLastError();
		return PSG_E_CUDA;
	}
	if (device < 0 || device >= ndev) return PSG_E_INVAL;
	psg_context *ctx = new psg_context();
	ctx->device = device;
	if (cudaSetDevice(device) != cudaSuccess ||
			cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
			cudaMalloc(&ctx->d_status, sizeof(uint32_t)) != cudaSuccess ||
			cudaMemset(ctx->d_status, 0, sizeof(uint32_t)) != cudaSuccess ||
			cudaMalloc(&ctx->d_counters, 32 * sizeof(unsigned long long)) != cudaSuccess ||
			cudaMemset(ctx->d_counters, 0, 32 * sizeof(unsigned long long)) != cudaSuccess ||
			cudaMalloc(&ctx->d_batch, sizeof(PsgBatchDev)) != cudaSuccess ||
			cudaDeviceGetAttribute(&ctx->sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
		cudaGetLastError();
		delete ctx;
		return PSG_E_CUDA;
	}
	ctx->stream = ctx->own_stream;
	for (auto &ev : ctx->ev) cudaEventCreate(&ev);
	psg_tune_cached(device, &ctx->tune);     // the device's tuned shapes, if any
	// reserve psg_step_evolve_noalloc's static buffer on this device now (its
	// module loads on the first lookup), not on its first call
	unsigned char *nb = nullptr;
	if (psg_noalloc_lookup(&nb) != 0) {
		psg_destroy(ctx);
		return PSG_E_CUDA;
	}
	*out = ctx;
	return PSG_OK;
}

static void free_particles(psg_context *ctx) {
	void *ptrs[] = {ctx->d_psml, ctx->d_mass, ctx->d_rho, ctx->d_yeMET, ctx->d_ie, ctx->d_flag,
		ctx->d_lambdaH, ctx->d_hits, ctx->d_lasthit, ctx->d_hstep, ctx->d_order, ctx->d_gcarry, ctx->d_ygrec,
		ctx->d_srcmark, ctx->d_lamHeI, ctx->d_lamHeII, ctx->d_ygrecHe1, ctx->d_ygrecHe2, ctx->d_gcarryHe1,
		ctx->d_gcarryHe2};
	for (void *p : ptrs) if (p) cudaFree(p);
	ctx->d_psml = nullptr; ctx->d_mass = ctx->d_rho = ctx->d_yeMET = ctx->d_ie = nullptr;
	ctx->d_flag = nullptr; ctx->d_lambdaH = nullptr; ctx->d_hits = nullptr; ctx->d_lasthit = nullptr;
	ctx->d_hstep = nullptr; ctx->d_order = nullptr; ctx->d_gcarry = nullptr; ctx->d_ygrec = nullptr;
	ctx->d_srcmark = nullptr; ctx->d_lamHeI = ctx->d_lamHeII = nullptr;
	ctx->d_ygrecHe1 = ctx->d_ygrecHe2 = nullptr;
	ctx->d_gcarryHe1 = ctx->d_gcarryHe2 = nullptr;
	ctx->rec_last = ctx->rec_last_R = 0;
	ctx->n = 0;
}

static void free_tree(psg_context *ctx) {
	void *ptrs[] = {ctx->d_cell_lo, ctx->d_cell_hi, ctx->d_wide_lo, ctx->d_wide_hi, ctx->d_leaf_psml, ctx->d_leaf_idx};
	for (void *p : ptrs) if (p) cudaFree(p);
	ctx->d_cell_lo = ctx->d_cell_hi = ctx->d_wide_lo = ctx->d_wide_hi = ctx->d_leaf_psml = nullptr;
	ctx->d_leaf_idx = nullptr;
	ctx->have_tree = 0;
}

extern "C" void psg_destroy(psg_context *ctx) {
	if (!ctx) return;
	cudaSetDevice(ctx->device);
	cudaStreamSynchronize(ctx->stream);
	free_particles(ctx);
	free_tree(ctx);
	if (ctx->d_ar) cudaFree(ctx->d_ar);
	if (ctx->d_ar_ni) cudaFree(ctx->d_ar_ni);
	if (ctx->d_xs) cudaFree(ctx->d_xs);
	if (ctx->d_kernel) cudaFree(ctx->d_kernel);
	if (ctx->d_status) cudaFree(ctx->d_status);
	if (ctx->d_counters) cudaFree(ctx->d_counters);
	if (ctx->d_batch) cudaFree(ctx->d_batch);
	psg_graphs_free(ctx);
	if (ctx->d_emit) cudaFree(ctx->d_emit);
	if (ctx->d_surr) cudaFree(ctx->d_surr);
	if (ctx->d_lte) cudaFree(ctx->d_lte);
	if (ctx->d_si) cudaFree(ctx->d_si);
	for (auto &b : ctx->scratch) if (b.p) cudaFree(b.p);
	for (auto &ev : ctx->ev) if (ev) cudaEventDestroy(ev);
	for (auto &ev : ctx->kev) if (ev) cudaEventDestroy(ev);
	cudaStreamDestroy(ctx->own_stream);
	delete ctx;
}

// ---- particle-state snapshot (autotuner trials, a recombination batch's undo) --
namespace {
struct StateArray {
	void *p;
	size_t item;
};
int state_arrays(psg_context *ctx, StateArray *out) {
	int k = 0;
	out[k++] = {ctx->d_lambdaH, sizeof(double)};
	out[k++] = {ctx->d_ie, sizeof(float)};
	out[k++] = {ctx->d_hits, sizeof(int32_t)};
	out[k++] = {ctx->d_lasthit, sizeof(int64_t)};
	out[k++] = {ctx->d_hstep, sizeof(float)};
	out[k++] = {ctx->d_gcarry, sizeof(double)};
	out[k++] = {ctx->d_ygrec, sizeof(float)};
	out[k++] = {ctx->d_srcmark, sizeof(int32_t)};
	out[k++] = {ctx->d_lamHeI, sizeof(double)};
	out[k++] = {ctx->d_lamHeII, sizeof(double)};
	out[k++] = {ctx->d_ygrecHe1, sizeof(float)};
	out[k++] = {ctx->d_ygrecHe2, sizeof(float)};
	out[k++] = {ctx->d_gcarryHe1, sizeof(double)};
	out[k++] = {ctx->d_gcarryHe2, sizeof(double)};
	return k;
}
}  // namespace

int psg_state_save(psg_context *ctx) {
	StateArray a[16];
	const int na = state_arrays(ctx, a);
	size_t total = 0;
	for (int i = 0; i < na; i++) total += (a[i].item * ctx->n + 255) & ~(size_t)255;
	char *snap = (char *)psg_scratch(ctx, S_SNAP, total);
	if (!snap) return PSG_E_NOMEM;
	for (int i = 0; i < na; i++) {
		const size_t b = a[i].item * ctx->n;
		if (a[i].p) PSG_CUDA(cudaMemcpyAsync(snap, a[i].p, b, cudaMemcpyDeviceToDevice, ctx->stream));
		snap += (b + 255) & ~(size_t)255;
	}
	return PSG_OK;
}

int psg_state_restore(psg_context *ctx) {
	StateArray a[16];
	const int na = state_arrays(ctx, a);
	char *snap = (char *)ctx->scratch[S_SNAP].p;
	if (!snap) return psg_fail(ctx, PSG_E_INVAL, "no saved state");
	for (int i = 0; i < na; i++) {
		const size_t b = a[i].item * ctx->n;
		if (a[i].p) PSG_CUDA(cudaMemcpyAsync(a[i].p, snap, b, cudaMemcpyDeviceToDevice, ctx->stream));
		snap += (b + 255) & ~(size_t)255;
	}
	return PSG_OK;
}

// ---- launch shapes ----------------------------------------------------------
namespace {
std::mutex g_tune_mutex;
psg_tune g_tune_cache[64];
bool g_tune_have[64];
int check_tune(const psg_tune *t) {
	if (t->trace_warps < 1 || t->trace_warps > 16) return 0;
	if (t->deposit_long < 32 || t->deposit_mid < t->deposit_long || t->deposit_mid > 1 << 20) return 0;
	if (t->update_minblocks != 1 && t->update_minblocks != 3 && t->update_minblocks != 4) return 0;
	if (t->run_short != 4 && t->run_short != 8 && t->run_short != 16) return 0;
	if (t->update_order != 0 && t->update_order != 1) return 0;
	return t->leaf_size == 8;
}
}  // namespace

bool psg_tune_cached(int device, psg_tune *t) {
	if (device < 0 || device >= 64) return false;
	std::lock_guard<std::mutex> lock(g_tune_mutex);
	if (!g_tune_have[device]) return false;
	*t = g_tune_cache[device];
	return true;
}

void psg_tune_store(int device, const psg_tune *t) {
	if (device < 0 || device >= 64) return;
	std::lock_guard<std::mutex> lock(g_tune_mutex);
	g_tune_cache[device] = *t;
	g_tune_have[device] = true;
}

extern "C" int psg_set_tune(psg_context *ctx, const psg_tune *tune) {
	if (!ctx) return PSG_E_INVAL;
	if (!tune || !check_tune(tune))
		return psg_fail(ctx, PSG_E_INVAL, "psg_set_tune: trace_warps 1-16, 32 <= deposit_long <= deposit_mid, "
				"update_minblocks 1, 3 or 4, leaf_size 8, run_short 4, 8 or 16, update_order 0 or 1");
	ctx->tune = *tune;
	return PSG_OK;
}

extern "C" int psg_get_tune(psg_context *ctx, psg_tune *tune) {
	if (!ctx || !tune) return PSG_E_INVAL;
	*tune = ctx->tune;
	return PSG_OK;
}

extern "C" const char *psg_last_error(const psg_context *ctx) {
	return ctx ? ctx->err : "no context";
}

extern "C" int psg_set_timing(psg_context *ctx, int on) {
	if (!ctx) return PSG_E_INVAL;
	PSG_CUDA(cudaSetDevice(ctx->device));
	if (on && !ctx->kev[0])
		for (auto &e : ctx->kev) PSG_CUDA(cudaEventCreate(&e));
	ctx->timing = on ? 1 : 0;
	return PSG_OK;
}

extern "C" int psg_set_stream(psg_context *ctx, void *stream) {
	if (!ctx) return PSG_E_INVAL;
	PSG_CUDA(cudaSetDevice(ctx->device));
	PSG_CUDA(cudaStreamSynchronize(ctx->stream));
	ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
	return PSG_OK;
}

extern "C" int psg_set_physics(psg_context *ctx, const psg_units *u, const psg_rate_table *ar,
		const psg_xs_table *xs, const double *kernel, int kernel_n, const psg_flags *flags) {
	if (!ctx) return PSG_E_INVAL;
	if (!u || !ar || !xs || !kernel || kernel_n <= 0 || !flags || ar->nrows < 2 || xs->nrows < 2)
		return psg_fail(ctx, PSG_E_INVAL, "psg_set_physics: missing or empty table");
	PSG_CUDA(cudaSetDevice(ctx->device));
	if (ctx->d_ar) cudaFree(ctx->d_ar);
	if (ctx->d_ar_ni) cudaFree(ctx->d_ar_ni);
	if (ctx->d_ar_all) cudaFree(ctx->d_ar_all);
	if (ctx->d_xs) cudaFree(ctx->d_xs);
	if (ctx->d_kernel) cudaFree(ctx->d_kernel);
	ctx->d_ar = ctx->d_xs = ctx->d_kernel = nullptr;
	ctx->d_ar_ni = nullptr;
	ctx->d_ar_all = nullptr;
	// rows of 16 doubles (one 128-byte line): log T, then the 15 rate columns
	const size_t nr = (size_t)ar->nrows;
	static_assert(PSG_AR_NCOLS + 1 == 16, "one rate row is one 128-byte line");
	double *rows = (double *)malloc(sizeof(double) * nr * 16);
	if (!rows) return psg_fail(ctx, PSG_E_NOMEM, "psg_set_physics: host allocation failed");
	for (size_t j = 0; j < nr; j++) {
		rows[16 * j] = ar->logT[j];
		for (int c = 0; c < PSG_AR_NCOLS; c++) rows[16 * j + 1 + c] = ar->col[c][j];
	}
	cudaError_t e1 = cudaMalloc(&ctx->d_ar, sizeof(double) * nr * 16);
	if (e1 == cudaSuccess) e1 = cudaMemcpy(ctx->d_ar, rows, sizeof(double) * nr * 16, cudaMemcpyHostToDevice);
	free(rows);
	PSG_CUDA(e1);
	// The non-isothermal right-hand side needs 7 columns at one log T: one
	// 64-byte row per table row, the 7 values and their slopes per unit log T
	// in FP32, so a lookup is four 16-byte loads. Linear interpolation from
	// value and slope is the same line as tabfun_get()'s two-point form.
	{
		// (an eighth column, alpha_B, for the recombination photons when
		// not on the spot: alpha_AB = fdim(alpha_A, alpha_B), solve.c:59)
		const int ncol = flags->on_the_spot ? 7 : 8;
		const int cols[8] = {PSG_AR_HI_CI, flags->on_the_spot ? PSG_AR_HII_RC_B : PSG_AR_HII_RC_A,
				flags->on_the_spot ? PSG_AR_HII_RCC_B : PSG_AR_HII_RCC_A, PSG_AR_HI_CEC, PSG_AR_HI_CIC,
				PSG_AR_E_BREMC, PSG_AR_E_COMPC, PSG_AR_HII_RC_B};
		float *ni = (float *)calloc(nr * 16, sizeof(float));
		if (!ni) return psg_fail(ctx, PSG_E_NOMEM, "psg_set_physics: host allocation failed");
		// internal-unit rates (1e-140 .. 1e-56) are far below FP32's range:
		// each column is stored divided by its largest magnitude
		for (int c = 0; c < 8; c++) ctx->ar_ni_scale[c] = 1.0;
		for (int c = 0; c < ncol; c++) {
			double m = 0.0;
			for (size_t j = 0; j < nr; j++) m = fmax(m, fabs(ar->col[cols[c]][j]));
			ctx->ar_ni_scale[c] = m > 0.0 ? m : 1.0;
		}
		for (size_t j = 0; j < nr; j++)
			for (int c = 0; c < ncol; c++) {
				const double sc = ctx->ar_ni_scale[c];
				const double v = ar->col[cols[c]][j] / sc;
				const double s = j + 1 < nr ? (ar->col[cols[c]][j + 1] / sc - v) * ar->step_inv : 0.0;
				ni[16 * j + c] = (float)v;
				ni[16 * j + 8 + c] = (float)s;
			}
		cudaError_t e2 = cudaMalloc(&ctx->d_ar_ni, sizeof(float) * nr * 16);
		if (e2 == cudaSuccess) e2 = cudaMemcpy(ctx->d_ar_ni, ni, sizeof(float) * nr * 16, cudaMemcpyHostToDevice);
		free(ni);
		PSG_CUDA(e2);
	}
	// The helium right-hand side reads up to 15 columns: the same FP32 value
	// and slope form, a (value, slope) pair per column, one 128-byte row.
	{
		float *all = (float *)calloc(nr * 32, sizeof(float));
		if (!all) return psg_fail(ctx, PSG_E_NOMEM, "psg_set_physics: host allocation failed");
		for (int c = 0; c < PSG_AR_NCOLS; c++) {
			double m = 0.0;
			for (size_t j = 0; j < nr; j++) m = fmax(m, fabs(ar->col[c][j]));
			ctx->ar_all_scale[c] = m > 0.0 ? m : 1.0;
			for (size_t j = 0; j < nr; j++) {
				const double v = ar->col[c][j] / ctx->ar_all_scale[c];
				const double s = j + 1 < nr ? (ar->col[c][j + 1] / ctx->ar_all_scale[c] - v) * ar->step_inv : 0.0;
				all[32 * j + 2 * c] = (float)v;
				all[32 * j + 2 * c + 1] = (float)s;
			}
		}
		cudaError_t e4 = cudaMalloc(&ctx->d_ar_all, sizeof(float) * nr * 32);
		if (e4 == cudaSuccess) e4 = cudaMemcpy(ctx->d_ar_all, all, sizeof(float) * nr * 32, cudaMemcpyHostToDevice);
		free(all);
		PSG_CUDA(e4);
	}
	const size_t nx = (size_t)xs->nrows;
	PSG_CUDA(cudaMalloc(&ctx->d_xs, sizeof(double) * nx * 4));
	PSG_CUDA(cudaMemcpy(ctx->d_xs, xs->eng, sizeof(double) * nx, cudaMemcpyHostToDevice));
	for (int s = 0; s < 3; s++)
		PSG_CUDA(cudaMemcpy(ctx->d_xs + (1 + s) * nx, xs->sigma[PSG_XS_HI + s], sizeof(double) * nx,
				cudaMemcpyHostToDevice));
	if (flags->secondary_ionization && !ctx->d_si) {
		const size_t ns = (size_t)3 * PSG_SECION_NE * PSG_SECION_NX;
		double *h = (double *)malloc(sizeof(double) * ns);
		if (!h) return psg_fail(ctx, PSG_E_NOMEM, "psg_set_physics: host allocation failed");
		psg_secion_table_build(u, h);
		cudaError_t e3 = cudaMalloc(&ctx->d_si, sizeof(double) * ns);
		if (e3 == cudaSuccess) e3 = cudaMemcpy(ctx->d_si, h, sizeof(double) * ns, cudaMemcpyHostToDevice);
		free(h);
		PSG_CUDA(e3);
	}
	PSG_CUDA(cudaMalloc(&ctx->d_kernel, sizeof(double) * kernel_n));
	PSG_CUDA(cudaMemcpy(ctx->d_kernel, kernel, sizeof(double) * kernel_n, cudaMemcpyHostToDevice));
	ctx->u = *u;
	ctx->flags = *flags;
	ctx->ar_nrows = ar->nrows;
	ctx->ar_min = ar->min;
	ctx->ar_step_inv = ar->step_inv;
	ctx->ar_step = ar->step;
	ctx->xs_nrows = xs->nrows;
	ctx->xs_min = xs->min;
	ctx->xs_step_inv = xs->step_inv;
	ctx->xs_cut_HI = xs->cut[PSG_XS_HI];
	ctx->xs_cut_HeI = xs->cut[PSG_XS_HEI];
	ctx->xs_cut_HeII = xs->cut[PSG_XS_HEII];
	ctx->kernel_n = kernel_n;
	if (!flags->on_the_spot) {
		const int rc = psg_build_lte(ctx, xs);
		if (rc) return rc;
	}
	ctx->have_physics = 1;
	return PSG_OK;
}

// lambdaH and yeMET from the snapshot's xHI and ye, psystem.c:340-356 with
// psys_set_lambdaH() psystem.h:156-160 (hydrogen-only branch).
// With helium the rest of the ye block beyond x_HII is helium's electrons
// first (psystem.c:350-357, psys_set_lambdaHe() psystem.h:161-170); with
// HOnly the helium fractions stay 0.
__global__ void k_init_particles(size_t n, const float *pos, const float *sml, const float *xHI,
		const float *ye, int helium, double hmf, float4 *psml, double *lambdaH, float *yeMET,
		double *lamHeI, double *lamHeII) {
	const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
	if (i >= n) return;
	psml[i] = make_float4(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], sml[i]);
	const double xhi = xHI[i];
	const double xhii = rn_dsub(1.0, xhi);
	double lam;
	if (xhi >= 1.0 || xhii <= 0.0) lam = 1.0;
	else if (xhi <= 0.0 || xhii >= 1.0) lam = 0.0;
	else lam = xhi;
	lambdaH[i] = lam;
	double yem = fdim((double)ye[i], xhii);
	double l1 = 0.0, l2 = 0.0;
	if (helium) {
		double x2 = yem * hmf / (1 - hmf) * 4;
		double x3 = fdim(x2, 1.0);
		x2 = fmin(1.0, x2);
		x3 = fmin(1.0 - x2, x3);
		const double x1 = 1.0 - x2 - x3;
		if (x1 >= 1.0 || (x2 + x3) <= 0.0) l1 = 1.0;
		else if (x1 <= 0.0 || (x2 + x3) >= 1.0) l1 = 0.0;
		else l1 = x1;
		if (x2 >= 1.0 || (x1 + x3) <= 0.0) l2 = 1.0;
		else if (x2 <= 0.0 || (x3 + x1) >= 1.0) l2 = 0.0;
		else l2 = x2;
		yem = fdim(yem, (x2 + 2 * x3) * (1 - hmf) / hmf * 0.25);
	}
	lamHeI[i] = l1;
	lamHeII[i] = l2;
	yeMET[i] = (float)yem;
}

// The architecture of the device code the runtime loaded for this library
// (one kernel stands for all: every .cu file is built with the same
// -gencode). No reference counterpart: a build check for the host.
extern "C" int psg_device_arch(psg_context *ctx, int *binary_version, int *ptx_version) {
	if (!ctx || !binary_version || !ptx_version) return PSG_E_INVAL;
	PSG_CUDA(cudaSetDevice(ctx->device));
	cudaFuncAttributes a;
	PSG_CUDA(cudaFuncGetAttributes(&a, k_init_particles));
	*binary_version = a.binaryVersion;
	*ptx_version = a.ptxVersion;
	return PSG_OK;
}

extern "C" int psg_load_particles(psg_context *ctx, const psg_particles *p) {
	if (!ctx) return PSG_E_INVAL;
	if (!p || p->n == 0 || !p->pos || !p->mass || !p->sml || !p->rho || !p->ie || !p->xHI || !p->ye)
		return psg_fail(ctx, PSG_E_INVAL, "psg_load_particles: missing array");
	if (p->n >= (size_t)PSG_INVALID_BIT)
		return psg_fail(ctx, PSG_E_OVERFLOW, "psg_load_particles: at most 2^31-1 particles");
	if (!(p->boxsize > 0))
		return psg_fail(ctx, PSG_E_INVAL, "psg_load_particles: boxsize must be positive");
	PSG_CUDA(cudaSetDevice(ctx->device));
	free_particles(ctx);
	free_tree(ctx);
	const size_t n = p->n;
	ctx->n = n;
	ctx->boxsize = p->boxsize;
	ctx->sat_frac = 0.0;       // a new field starts on the deposit's common form
	PSG_CUDA(cudaMalloc(&ctx->d_psml, sizeof(float4) * n));
	PSG_CUDA(cudaMalloc(&ctx->d_mass, sizeof(float) * n));
	PSG_CUDA(cudaMalloc(&ctx->d_rho, sizeof(float) * n));
	PSG_CUDA(cudaMalloc(&ctx->d_yeMET, sizeof(float) * n));
	PSG_CUDA(cudaMalloc(&ctx->d_ie, sizeof(float) * n));
	PSG_CUDA(cudaMalloc(&ctx->d_flag, n));
	PSG_CUDA(cudaMalloc(&ctx->d_lambdaH, sizeof(double) * n));
	PSG_CUDA(cudaMalloc(&ctx->d_hits, sizeof(int32_t) * n));
	PSG_CUDA(cudaMalloc(&ctx->d_lasthit, sizeof(int64_t) * n));
	PSG_CUDA(cudaMalloc(&ctx->d_hstep, sizeof(float) * n));
	PSG_CUDA(cudaMalloc(&ctx->d_gcarry, sizeof(double) * n));
	PSG_CUDA(cudaMalloc(&ctx->d_ygrec, sizeof(float) * n));
	PSG_CUDA(cudaMalloc(&ctx->d_srcmark, sizeof(int32_t) * n));
	PSG_CUDA(cudaMalloc(&ctx->d_lamHeI, sizeof(double) * n));
	PSG_CUDA(cudaMalloc(&ctx->d_lamHeII, sizeof(double) * n));
	PSG_CUDA(cudaMalloc(&ctx->d_ygrecHe1, sizeof(float) * n));
	PSG_CUDA(cudaMalloc(&ctx->d_ygrecHe2, sizeof(float) * n));
	PSG_CUDA(cudaMalloc(&ctx->d_gcarryHe1, sizeof(double) * n));
	PSG_CUDA(cudaMalloc(&ctx->d_gcarryHe2, sizeof(double) * n));
	float *d_pos = (float *)psg_scratch(ctx, S_MISC, sizeof(float) * n * 7);
	if (!d_pos) return PSG_E_NOMEM;
	float *d_sml = d_pos + 3 * n, *d_xHI = d_pos + 4 * n, *d_ye = d_pos + 5 * n;
	cudaStream_t s = ctx->stream;
	PSG_CUDA(cudaMemcpyAsync(d_pos, p->pos, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, s));
	PSG_CUDA(cudaMemcpyAsync(d_sml, p->sml, sizeof(float) * n, cudaMemcpyHostToDevice, s));
	PSG_CUDA(cudaMemcpyAsync(d_xHI, p->xHI, sizeof(float) * n, cudaMemcpyHostToDevice, s));
	PSG_CUDA(cudaMemcpyAsync(d_ye, p->ye, sizeof(float) * n, cudaMemcpyHostToDevice, s));
	PSG_CUDA(cudaMemcpyAsync(ctx->d_mass, p->mass, sizeof(float) * n, cudaMemcpyHostToDevice, s));
	PSG_CUDA(cudaMemcpyAsync(ctx->d_rho, p->rho, sizeof(float) * n, cudaMemcpyHostToDevice, s));
	PSG_CUDA(cudaMemcpyAsync(ctx->d_ie, p->ie, sizeof(float) * n, cudaMemcpyHostToDevice, s));
	if (p->flag) PSG_CUDA(cudaMemcpyAsync(ctx->d_flag, p->flag, n, cudaMemcpyHostToDevice, s));
	else PSG_CUDA(cudaMemsetAsync(ctx->d_flag, 0, n, s));
	PSG_CUDA(cudaMemsetAsync(ctx->d_hits, 0, sizeof(int32_t) * n, s));
	PSG_CUDA(cudaMemsetAsync(ctx->d_lasthit, 0, sizeof(int64_t) * n, s));
	PSG_CUDA(cudaMemsetAsync(ctx->d_hstep, 0, sizeof(float) * n, s));
	PSG_CUDA(cudaMemsetAsync(ctx->d_gcarry, 0, sizeof(double) * n, s));
	PSG_CUDA(cudaMemsetAsync(ctx->d_ygrec, 0, sizeof(float) * n, s));
	PSG_CUDA(cudaMemsetAsync(ctx->d_ygrecHe1, 0, sizeof(float) * n, s));
	PSG_CUDA(cudaMemsetAsync(ctx->d_ygrecHe2, 0, sizeof(float) * n, s));
	PSG_CUDA(cudaMemsetAsync(ctx->d_gcarryHe1, 0, sizeof(double) * n, s));
	PSG_CUDA(cudaMemsetAsync(ctx->d_gcarryHe2, 0, sizeof(double) * n, s));
	PSG_CUDA(cudaMemsetAsync(ctx->d_srcmark, 0xff, sizeof(int32_t) * n, s));
	const int bs = 256;
	k_init_particles<<<(unsigned)((n + bs - 1) / bs), bs, 0, s>>>(n, d_pos, d_sml, d_xHI, d_ye,
			ctx->have_physics && !ctx->flags.h_only, ctx->u.hmf, ctx->d_psml, ctx->d_lambdaH, ctx->d_yeMET,
			ctx->d_lamHeI, ctx->d_lamHeII);
	PSG_CHECK_LAUNCH();
	PSG_CUDA(cudaStreamSynchronize(s));
	return PSG_OK;
}

// ---- particle order ----------------------------------------------------------
// After psg_build_tree the per-particle arrays are kept in the tree's leaf
// order (internal position k holds the caller's particle d_order[k]), so the
// particles a ray meets one after another sit next to each other in memory.
// The caller only ever sees its own order: the state calls and the hit lists
// map through d_order.
template <typename T>
__global__ void k_gather(size_t n, const uint32_t *__restrict__ g, const T *__restrict__ in, T *__restrict__ out) {
	const size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
	if (k < n) out[k] = in[g[k]];
}
template <typename T>
__global__ void k_scatter(size_t n, const uint32_t *__restrict__ g, const T *__restrict__ in, T *__restrict__ out) {
	const size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
	if (k < n) out[g[k]] = in[k];
}

template <typename T>
static int permute_array(psg_context *ctx, T *&arr, const uint32_t *g) {
	const size_t n = ctx->n;
	T *out = nullptr;
	PSG_CUDA(cudaMalloc(&out, sizeof(T) * n));
	k_gather<T><<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(n, g, arr, out);
	const cudaError_t e = cudaGetLastError();
	if (e != cudaSuccess) {
		cudaFree(out);
		return psg_cuda_fail(ctx, e, "k_gather", __FILE__, __LINE__);
	}
	PSG_CUDA(cudaStreamSynchronize(ctx->stream));
	PSG_CUDA(cudaFree(arr));
	arr = out;
	return PSG_OK;
}

int psg_permute_particles(psg_context *ctx, const uint32_t *g) {
	int rc = 0;
	if ((rc = permute_array(ctx, ctx->d_psml, g)) || (rc = permute_array(ctx, ctx->d_mass, g)) ||
			(rc = permute_array(ctx, ctx->d_rho, g)) || (rc = permute_array(ctx, ctx->d_yeMET, g)) ||
			(rc = permute_array(ctx, ctx->d_ie, g)) || (rc = permute_array(ctx, ctx->d_flag, g)) ||
			(rc = permute_array(ctx, ctx->d_lambdaH, g)) || (rc = permute_array(ctx, ctx->d_hits, g)) ||
			(rc = permute_array(ctx, ctx->d_lasthit, g)) || (rc = permute_array(ctx, ctx->d_hstep, g)) ||
			(rc = permute_array(ctx, ctx->d_gcarry, g)) || (rc = permute_array(ctx, ctx->d_ygrec, g)) ||
			(rc = permute_array(ctx, ctx->d_srcmark, g)) || (rc = permute_array(ctx, ctx->d_lamHeI, g)) ||
			(rc = permute_array(ctx, ctx->d_lamHeII, g)) || (rc = permute_array(ctx, ctx->d_ygrecHe1, g)) ||
			(rc = permute_array(ctx, ctx->d_ygrecHe2, g)) || (rc = permute_array(ctx, ctx->d_gcarryHe1, g)) ||
			(rc = permute_array(ctx, ctx->d_gcarryHe2, g)))
		return rc;
	// the caller index of every new position: through the previous order
	const size_t n = ctx->n;
	uint32_t *order = nullptr;
	PSG_CUDA(cudaMalloc(&order, sizeof(uint32_t) * n));
	if (ctx->d_order) {
		k_gather<uint32_t><<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(n, g, ctx->d_order, order);
		PSG_CHECK_LAUNCH();
		PSG_CUDA(cudaStreamSynchronize(ctx->stream));
		PSG_CUDA(cudaFree(ctx->d_order));
	} else {
		PSG_CUDA(cudaMemcpyAsync(order, g, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, ctx->stream));
		PSG_CUDA(cudaStreamSynchronize(ctx->stream));
	}
	ctx->d_order = order;
	return PSG_OK;
}

// device array (internal order) -> host array (caller order)
template <typename T>
static int to_caller(psg_context *ctx, T *host, const T *dev) {
	const size_t n = ctx->n;
	cudaStream_t s = ctx->stream;
	if (!ctx->d_order) {
		PSG_CUDA(cudaMemcpyAsync(host, dev, sizeof(T) * n, cudaMemcpyDeviceToHost, s));
		return PSG_OK;
	}
	T *tmp = (T *)psg_scratch(ctx, S_MAP, sizeof(T) * n);
	if (!tmp) return PSG_E_NOMEM;
	k_scatter<T><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, ctx->d_order, dev, tmp);
	PSG_CHECK_LAUNCH();
	PSG_CUDA(cudaMemcpyAsync(host, tmp, sizeof(T) * n, cudaMemcpyDeviceToHost, s));
	PSG_CUDA(cudaStreamSynchronize(s));
	return PSG_OK;
}

// host array (caller order) -> device array (internal order)
template <typename T>
static int from_caller(psg_context *ctx, T *dev, const T *host) {
	const size_t n = ctx->n;
	cudaStream_t s = ctx->stream;
	if (!ctx->d_order) {
		PSG_CUDA(cudaMemcpyAsync(dev, host, sizeof(T) * n, cudaMemcpyHostToDevice, s));
		return PSG_OK;
	}
	T *tmp = (T *)psg_scratch(ctx, S_MAP, sizeof(T) * n);
	if (!tmp) return PSG_E_NOMEM;
	PSG_CUDA(cudaMemcpyAsync(tmp, host, sizeof(T) * n, cudaMemcpyHostToDevice, s));
	k_gather<T><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, ctx->d_order, tmp, dev);
	PSG_CHECK_LAUNCH();
	PSG_CUDA(cudaStreamSynchronize(s));
	return PSG_OK;
}

extern "C" int psg_get_state(psg_context *ctx, double *lambdaH, float *ie, int32_t *hits,
		int64_t *lasthit) {
	if (!ctx) return PSG_E_INVAL;
	if (!ctx->n) return psg_fail(ctx, PSG_E_INVAL, "psg_get_state: no particles loaded");
	PSG_CUDA(cudaSetDevice(ctx->device));
	int rc = 0;
	if (lambdaH && (rc = to_caller(ctx, lambdaH, ctx->d_lambdaH))) return rc;
	if (ie && (rc = to_caller(ctx, ie, ctx->d_ie))) return rc;
	if (hits && (rc = to_caller(ctx, hits, ctx->d_hits))) return rc;
	if (lasthit && (rc = to_caller(ctx, lasthit, ctx->d_lasthit))) return rc;
	PSG_CUDA(cudaStreamSynchronize(ctx->stream));
	return PSG_OK;
}

extern "C" int psg_set_state(psg_context *ctx, const double *lambdaH, const float *ie,
		const int64_t *lasthit) {
	if (!ctx) return PSG_E_INVAL;
	if (!ctx->n) return psg_fail(ctx, PSG_E_INVAL, "psg_set_state: no particles loaded");
	PSG_CUDA(cudaSetDevice(ctx->device));
	int rc = 0;
	if (lambdaH && (rc = from_caller(ctx, ctx->d_lambdaH, lambdaH))) return rc;
	if (ie && (rc = from_caller(ctx, ctx->d_ie, ie))) return rc;
	if (lasthit && (rc = from_caller(ctx, ctx->d_lasthit, lasthit))) return rc;
	PSG_CUDA(cudaStreamSynchronize(ctx->stream));
	return PSG_OK;
}

extern "C" int psg_set_hits(psg_context *ctx, const int32_t *hits) {
	if (!ctx) return PSG_E_INVAL;
	if (!ctx->n || !hits) return psg_fail(ctx, PSG_E_INVAL, "psg_set_hits: no particles or no counters");
	PSG_CUDA(cudaSetDevice(ctx->device));
	const int rc = from_caller(ctx, ctx->d_hits, hits);
	if (rc) return rc;
	PSG_CUDA(cudaStreamSynchronize(ctx->stream));
	return PSG_OK;
}

extern "C" int psg_get_he_state(psg_context *ctx, double *lambdaHeI, double *lambdaHeII, float *yeMET,
		float *yGrecHeII, float *yGrecHeIII) {
	if (!ctx) return PSG_E_INVAL;
	if (!ctx->n) return psg_fail(ctx, PSG_E_INVAL, "psg_get_he_state: no particles loaded");
	PSG_CUDA(cudaSetDevice(ctx->device));
	int rc = 0;
	if (lambdaHeI && (rc = to_caller(ctx, lambdaHeI, ctx->d_lamHeI))) return rc;
	if (lambdaHeII && (rc = to_caller(ctx, lambdaHeII, ctx->d_lamHeII))) return rc;
	if (yeMET && (rc = to_caller(ctx, yeMET, ctx->d_yeMET))) return rc;
	if (yGrecHeII && (rc = to_caller(ctx, yGrecHeII, ctx->d_ygrecHe1))) return rc;
	if (yGrecHeIII && (rc = to_caller(ctx, yGrecHeIII, ctx->d_ygrecHe2))) return rc;
	PSG_CUDA(cudaStreamSynchronize(ctx->stream));
	return PSG_OK;
}

extern "C" int psg_set_he_state(psg_context *ctx, const double *lambdaHeI, const double *lambdaHeII,
		const float *yGrecHeII, const float *yGrecHeIII) {
	if (!ctx) return PSG_E_INVAL;
	if (!ctx->n) return psg_fail(ctx, PSG_E_INVAL, "psg_set_he_state: no particles loaded");
	PSG_CUDA(cudaSetDevice(ctx->device));
	int rc = 0;
	if (lambdaHeI && (rc = from_caller(ctx, ctx->d_lamHeI, lambdaHeI))) return rc;
	if (lambdaHeII && (rc = from_caller(ctx, ctx->d_lamHeII, lambdaHeII))) return rc;
	if (yGrecHeII && (rc = from_caller(ctx, ctx->d_ygrecHe1, yGrecHeII))) return rc;
	if (yGrecHeIII && (rc = from_caller(ctx, ctx->d_ygrecHe2, yGrecHeIII))) return rc;
	PSG_CUDA(cudaStreamSynchronize(ctx->stream));
	return PSG_OK;
}

extern "C" int psg_get_rec_state(psg_context *ctx, float *yGrecHII, int32_t *srcmark) {
	if (!ctx) return PSG_E_INVAL;
	if (!ctx->n) return psg_fail(ctx, PSG_E_INVAL, "psg_get_rec_state: no particles loaded");
	PSG_CUDA(cudaSetDevice(ctx->device));
	int rc = 0;
	if (yGrecHII && (rc = to_caller(ctx, yGrecHII, ctx->d_ygrec))) return rc;
	if (srcmark && (rc = to_caller(ctx, srcmark, ctx->d_srcmark))) return rc;
	PSG_CUDA(cudaStreamSynchronize(ctx->stream));
	return PSG_OK;
}

extern "C" int psg_set_rec_state(psg_context *ctx, const float *yGrecHII, const int32_t *srcmark) {
	if (!ctx) return PSG_E_INVAL;
	if (!ctx->n) return psg_fail(ctx, PSG_E_INVAL, "psg_set_rec_state: no particles loaded");
	PSG_CUDA(cudaSetDevice(ctx->device));
	int rc = 0;
	if (yGrecHII && (rc = from_caller(ctx, ctx->d_ygrec, yGrecHII))) return rc;
	if (srcmark && (rc = from_caller(ctx, ctx->d_srcmark, srcmark))) return rc;
	PSG_CUDA(cudaStreamSynchronize(ctx->stream));
	return PSG_OK;
}

extern "C" int psg_write_output(psg_context *ctx, const char *filename, const psg_snapshot *meta) {
	if (!ctx) return PSG_E_INVAL;
	if (!filename || !meta || meta->ngas != ctx->n || !ctx->n)
		return psg_fail(ctx, PSG_E_INVAL, "psg_write_output: meta->ngas must equal the loaded particle count");
	if (!ctx->have_physics) return psg_fail(ctx, PSG_E_INVAL, "psg_write_output: set physics first");
	PSG_CUDA(cudaSetDevice(ctx->device));
	const size_t n = ctx->n;
	std::vector<float4> psml(n);
	std::vector<float> pos(3 * n), sml(n), mass(n), rho(n), ie(n), xHI(n), ye(n), xHeI(n), xHeII(n), ygrec(n);
	std::vector<double> lam(n), l1(n), l2(n);
	std::vector<int32_t> hits(n);
	std::vector<int64_t> lasthit(n), ids;
	int rc = 0;
	if ((rc = to_caller(ctx, psml.data(), ctx->d_psml)) || (rc = to_caller(ctx, mass.data(), ctx->d_mass)) ||
			(rc = to_caller(ctx, rho.data(), ctx->d_rho)) || (rc = to_caller(ctx, ie.data(), ctx->d_ie)) ||
			(rc = to_caller(ctx, lam.data(), ctx->d_lambdaH)) || (rc = to_caller(ctx, hits.data(), ctx->d_hits)) ||
			(rc = to_caller(ctx, lasthit.data(), ctx->d_lasthit)) || (rc = to_caller(ctx, l1.data(), ctx->d_lamHeI)) ||
			(rc = to_caller(ctx, l2.data(), ctx->d_lamHeII)) || (rc = to_caller(ctx, ygrec.data(), ctx->d_ygrec)))
		return rc;
	PSG_CUDA(cudaStreamSynchronize(ctx->stream));
	// psys_ye() psystem.h:177 (lambda_to_ye() psystem.h:134-138): with
	// HOnly both helium fractions are 0, i.e. helium frozen fully ionised
	for (size_t i = 0; i < n; i++) {
		pos[3 * i] = psml[i].x;
		pos[3 * i + 1] = psml[i].y;
		pos[3 * i + 2] = psml[i].z;
		sml[i] = psml[i].w;
		xHI[i] = (float)lam[i];
		xHeI[i] = (float)l1[i];
		xHeII[i] = (float)l2[i];
		ye[i] = (float)((1.0 - lam[i]) + ctx->u.hemf / ctx->u.hmf * 0.25 * (l2[i] + 2 * (1.0 - l2[i] - l1[i])));
	}
	psg_snapshot s = *meta;
	if (!s.id) {
		ids.resize(n);
		for (size_t i = 0; i < n; i++) ids[i] = (int64_t)i;
		s.id = ids.data();
	}
	s.pos = pos.data();
	s.sml = sml.data();
	s.mass = mass.data();
	s.rho = rho.data();
	s.ie = ie.data();
	s.xHI = xHI.data();
	s.ye = ye.data();
	s.xHeI = xHeI.data();
	s.xHeII = xHeII.data();
	s.gammaHI = ygrec.data();      // the block holds yGrecHII (psystem.c:653)
	s.lasthit = lasthit.data();
	s.hits = hits.data();
	if (s.boxsize == 0.0) s.boxsize = ctx->boxsize;
	rc = psg_snapshot_write(filename, &s);
	if (rc) return psg_fail(ctx, rc, "psg_write_output: writing %s failed", filename);
	return PSG_OK;
}
