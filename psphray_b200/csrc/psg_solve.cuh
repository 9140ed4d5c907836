// Per-particle ionisation update on the device; replaces step_evolve()
// solve.c:317 (LSODA over the 7-variable system of solve.c:76-141).
//
// Hydrogen-only, so only lambdaH (= xHI) and, when not isothermal, the
// internal energy ie move. Normalised time s in [0,1] as in the reference
// (every derivative multiplied by the step length, solve.c:120-121).
//
// Isothermal: with ye = 1 + m - lambda (m = yeMET plus the frozen helium
// electrons), d(lambda)/ds = -g + tau*ye*(alpha*(1-lambda) - gamma*lambda) is
// a Riccati equation with constant coefficients,
//     d(lambda)/ds = a*lambda^2 - b*lambda + c,
// solved exactly about its stable root p1 in FP64, carried in lambda = 1-x so
// it stays accurate near full ionisation:
//     y(1) = y0*e^-k / (1 - a*y0*phi(k)),  y = lambda - p1,
//     k = sqrt(q^2 + 4*a*g), q = tau*(gamma*(1+m) + alpha*m), phi = (1-e^-k)/k,
//     p1 = 2c/(b + k).
// Not isothermal: adaptive Dormand-Prince 5(4) in FP64 over (lambda, ie).
//
// Recombination photons (onTheSpot = false): the case-A rate drives lambda
// and the recombination photons per H, d(yGrecHII)/ds = tau*alpha_AB*ye*x_HII
// (solve.c:83-86, alpha_AB = fdim(alpha_A, alpha_B)), are integrated beside
// it. Nothing depends on them, so the integrators carry them as a
// quadrature over the same stages (REC template flag), outside the error
// control; the isothermal closed form integrates them exactly:
//     int_0^1 lambda ds = p1 + y0*phi(k)*L(z),  z = a*y0*phi(k),
//     L(z) = -log(1-z)/z,
//     int_0^1 lambda^2 ds = (lambda(1) - lambda0 + b*int lambda - c)/a
// (the Riccati equation itself, a*lambda^2 = lambda' + b*lambda - c).
#pragma once

#include "psg_internal.cuh"

struct PhysParams {
	const double *ar;      // [ar_nrows][16]: log T, then the PSG_AR_* columns
	const float4 *ar_ni;   // [ar_nrows][4]: the right-hand side's 7 rates (+ alpha_B when not
	                       // on the spot), values and slopes
	double ar_ni_scale[8]; // ... each column divided by its largest magnitude
	const float2 *ar_all;  // [ar_nrows][16]: (value, slope) of all 15 columns (helium)
	double ar_all_scale[PSG_AR_NCOLS];
	int ar_nrows;
	double ar_min, ar_step_inv, ar_step;
	float ar_min_f, ar_step_inv_f, ar_step_f;   // the same in FP32 (the explicit stages' lookups)
	const double *xs;      // [4][xs_nrows]: energy, sigma_HI, sigma_HeI, sigma_HeII
	int xs_nrows;
	double xs_min, xs_step_inv, xs_cut_HI, xs_cut_HeI, xs_cut_HeII;
	const double *kernel;
	int kernel_n;
	double H_PER_MASS, HI_ENERGY, MPROTON_OVER_BOLTZMANN, BOLTZMANN_OVER_MPROTON, hmf, hemf;
	double he_e;           // helium electrons per H, helium frozen (psystem.h:134-137)
	int isothermal, on_the_spot, adiabatic, euler;
	float *ygrec;          // yGrecHII per particle (leaf order), when not on the spot
	// helium (h_only = 0) and secondary ionisation
	int h_only, secondary;
	double HE_PER_MASS, HEI_ENERGY, HEII_ENERGY;
	double *lamHeI, *lamHeII;
	float *ygrecHe1, *ygrecHe2;   // yGrecHeII, yGrecHeIII, when not on the spot
	double *gcarry, *gcarryHe1, *gcarryHe2;   // photons an explicit step left (helium ticks)
	const double *si;      // [3][PSG_SECION_NE][PSG_SECION_NX]: PhiHI, PhiHeI, Eh
	double si_min1, si_step1, si_step1_inv, si_min2, si_step2, si_step2_inv;
};

PhysParams psg_phys_params(const psg_context *ctx);

// tabfun_get() tabfun.c:38-58
__device__ __forceinline__ double tab_get(int nrows, double min, double step_inv,
		const double *__restrict__ x, const double *__restrict__ y, double v) {
	const long long idx = (long long)rn_dmul(rn_dsub(v, min), step_inv);
	if (idx < 0) return y[0];
	if (idx >= nrows - 1) return y[nrows - 1];
	const double lw = rn_dsub(x[idx + 1], v);
	const double rw = rn_dsub(v, x[idx]);
	return rn_dmul(rn_dadd(rn_dmul(lw, y[idx]), rn_dmul(rw, y[idx + 1])), step_inv);
}

// ar_get() atomic-rate.c:89 for several columns at one log T: the row index
// and the interpolation weights of tabfun_get() are computed once.
struct RateAt {
	const double *r0, *r1;
	double lw, rw, step_inv;
	int clamp;            // 0 interpolate, 1 first row, 2 last row
	__device__ __forceinline__ double operator()(int col) const {
		if (clamp == 1) return r0[1 + col];
		if (clamp == 2) return r1[1 + col];
		return rn_dmul(rn_dadd(rn_dmul(lw, r0[1 + col]), rn_dmul(rw, r1[1 + col])), step_inv);
	}
};

__device__ __forceinline__ RateAt rates_at(const PhysParams &P, double logT) {
	RateAt a;
	a.step_inv = P.ar_step_inv;
	const long long idx = (long long)rn_dmul(rn_dsub(logT, P.ar_min), P.ar_step_inv);
	if (idx < 0) {
		a.clamp = 1;
		a.r0 = a.r1 = P.ar;
		a.lw = a.rw = 0.0;
	} else if (idx >= P.ar_nrows - 1) {
		a.clamp = 2;
		a.r0 = a.r1 = P.ar + (size_t)(P.ar_nrows - 1) * 16;
		a.lw = a.rw = 0.0;
	} else {
		a.clamp = 0;
		a.r0 = P.ar + (size_t)idx * 16;
		a.r1 = a.r0 + 16;
		a.lw = rn_dsub(a.r1[0], logT);
		a.rw = rn_dsub(logT, a.r0[0]);
	}
	return a;
}

__device__ __forceinline__ double ar_get(const PhysParams &P, int col, double logT) {
	return rates_at(P, logT)(col);
}

// xs_get() atomic-rate.c:126-131 for HI
__device__ __forceinline__ double xs_get_HI(const PhysParams &P, double freq) {
	if (freq < P.xs_cut_HI) return 0.0;
	return tab_get(P.xs_nrows, P.xs_min, P.xs_step_inv, P.xs, P.xs + P.xs_nrows, freq);
}

// sph_depth() sph-depth.c:26-33
__device__ __forceinline__ double sph_depth(const PhysParams &P, double r_h) {
	const double x = rn_dmul((double)P.kernel_n, r_h);
	if (!(x < (double)P.kernel_n) || !(x > -1.0)) return 0.0;
	const int n = (int)x;
	if (n < P.kernel_n && n >= 0) return P.kernel[n];
	return 0.0;
}

// ieye2T() / Tye2ie() config.h:106-114
__device__ __forceinline__ double ieye2T(const PhysParams &P, double ie, double ye) {
	const double den = rn_dadd(rn_dadd(rn_dmul(P.hemf, 0.25), P.hmf), rn_dmul(P.hmf, ye));
	return __ddiv_rn(rn_dmul(__ddiv_rn(rn_dmul(P.MPROTON_OVER_BOLTZMANN, ie), den), 2.0), 3.0);
}
__device__ __forceinline__ double Tye2ie(const PhysParams &P, double T, double ye) {
	const double den = rn_dadd(rn_dadd(rn_dmul(P.hemf, 0.25), P.hmf), rn_dmul(P.hmf, ye));
	return rn_dmul(__ddiv_rn(rn_dmul(rn_dmul(T, P.BOLTZMANN_OVER_MPROTON), den), 2.0), 3.0);
}

__device__ __forceinline__ double phi_k(double k) {
	if (k > 1e-6) return -expm1(-k) / k;
	return 1.0 - k * (0.5 - k / 6.0);
}

// lambda(1); with I1 != NULL also int_0^1 lambda ds.
__device__ __forceinline__ double riccati_step(double lam0, double a, double b, double q, double c, double g,
		double *I1 = nullptr) {
	if (!(a > 0.0)) {
		if (b > 0.0) {
			const double eq = c / b;
			if (I1) *I1 = eq + (lam0 - eq) * phi_k(b);
			return eq + (lam0 - eq) * exp(-b);
		}
		if (I1) *I1 = lam0 + 0.5 * c;
		return lam0 + c;
	}
	const double k = sqrt(q * q + 4.0 * a * g);
	const double p1 = 2.0 * c / (b + k);
	const double y0 = lam0 - p1;
	const double ph = phi_k(k);
	if (I1) {
		const double z = a * y0 * ph;
		const double L = fabs(z) < 1e-4 ? 1.0 + z * (0.5 + z * (1.0 / 3.0 + 0.25 * z)) : -log1p(-z) / z;
		*I1 = p1 + y0 * ph * L;
	}
	return p1 + y0 * exp(-k) / (1.0 - a * y0 * ph);
}

// Recombination photons per H of one isothermal step: tau*alpha_AB times
// int_0^1 ye*x_HII ds, ye*x_HII = (1+m-lambda)(1-lambda), from the closed
// form's integrals (ar = alpha_AB/(alpha+gamma), the step's tau cancels).
__device__ __forceinline__ double riccati_rec(double lam0, double lam1, double I1, double a, double b, double c,
		double m, double tau_ab, double ar) {
	if (!(a > 0.0)) return 0.0;
	return tau_ab * ((1.0 + m) - (2.0 + m) * I1) + ar * (lam1 - lam0 + b * I1 - c);
}

struct RhsCtx {
	double yeMET, g, heat, time, nH, T;
	double nHt;                  // nH*time: rates per unit normalised time
	double hpt;                  // H_PER_MASS*time
	double T_num;                // MPROTON_OVER_BOLTZMANN*2/3: T = T_num*ie/(T_den0 + hmf*ye)
	double T_den0;               // hemf/4 + hmf
};

__device__ __forceinline__ RhsCtx make_rhs_ctx(const PhysParams &P, double yeMET, double g, double heat,
		double time, double nH, double T) {
	RhsCtx c;
	c.yeMET = yeMET; c.g = g; c.heat = heat; c.time = time; c.nH = nH; c.T = T;
	c.nHt = nH * time;
	c.hpt = P.H_PER_MASS * time;
	c.T_num = P.MPROTON_OVER_BOLTZMANN * 2.0 / 3.0;
	c.T_den0 = P.hemf * 0.25 + P.hmf;
	return c;
}

// function() solve.c:76-141, hydrogen-only branch, for the integrators (not
// isothermal): the same equations with the step length folded into the
// rates, and fused multiply-adds (the last bits of an integrator's stage do
// not matter; the isothermal closed form keeps the reference's roundings).
// With REC, *rec receives d(yGrecHII)/ds. With T32 (the explicit
// integrator's stages, not isothermal) the way from the state to the rates
// is FP32: the temperature with the fast divide, its logarithm with the
// fast log10 (a few ulp; the rate table is interpolated linearly, so an
// error e in log T moves a rate by its slope times e, about 1e-5 of itself
// at the steepest rows, the same order as FP32's own rounding of log T), the
// row and weight, and the interpolation of the FP32 table values; each rate
// is then scaled and combined in FP64, and the state and its derivatives
// stay FP64. Without it (finite-difference Jacobians, residual checks, the
// explicit build's steps) the lookup is FP64.
template <bool REC = false, bool T32 = false>
__device__ __forceinline__ void rhs(const PhysParams &P, const RhsCtx &cx, const double x[2], double dx[2],
		double *rec = nullptr) {
	const double xHI = x[0], xHII = 1.0 - x[0];
	const double ye = xHII + P.he_e + cx.yeMET;
	// the row of tabfun_get() and the offset into it (clamped rows, a NaN
	// temperature included: offset 0)
	long long idx;
	double du = 0.0;
	float duf = 0.0f;
	if (T32) {
		const float Tf = P.isothermal ? (float)cx.T
				: __fdividef((float)cx.T_num * (float)x[1], (float)__fma_rn(P.hmf, ye, cx.T_den0));
		const float lT = __log10f(Tf);
		const float uf = (lT - P.ar_min_f) * P.ar_step_inv_f;
		const int i = (int)uf;       // truncation; a NaN converts to 0, caught by uf == uf
		if (!(uf == uf) || i < 0) {
			idx = 0;
		} else if (i >= P.ar_nrows - 1) {
			idx = P.ar_nrows - 1;
		} else {
			idx = i;
			duf = lT - __fmaf_rn((float)i, P.ar_step_f, P.ar_min_f);
		}
	} else {
		const double logT = log10(P.isothermal ? cx.T : cx.T_num * x[1] / __fma_rn(P.hmf, ye, cx.T_den0));
		idx = (long long)((logT - P.ar_min) * P.ar_step_inv);
		if (idx < 0) {
			idx = 0;
		} else if (idx >= P.ar_nrows - 1) {
			idx = P.ar_nrows - 1;
		} else {
			du = logT - __fma_rn((double)idx, P.ar_step, P.ar_min);
		}
	}
	const float4 *row = P.ar_ni + 4 * idx;
	const float4 v0 = row[0], v1 = row[1], s0 = row[2], s1 = row[3];
#define PSG_LIN(v, s, c)                                                                                  \
	((T32 ? (double)__fmaf_rn((s), duf, (v)) : __fma_rn((double)(s), du, (double)(v))) * P.ar_ni_scale[c])
	const double gamma = PSG_LIN(v0.x, s0.x, 0) * cx.nHt;
	const double alpha = PSG_LIN(v0.y, s0.y, 1) * cx.nHt;       // case B on the spot, else A
	dx[0] = __fma_rn(ye, __fma_rn(alpha, xHII, -gamma * xHI), -cx.g);
	if (REC) {
		const double alphaB = PSG_LIN(v1.w, s1.w, 7) * cx.nHt;
		*rec = fdim(alpha, alphaB) * ye * xHII;
	}
	if (P.isothermal || P.adiabatic) {
		dx[1] = 0.0;
	} else {
		const double ion = PSG_LIN(v0.z, s0.z, 2) + PSG_LIN(v1.y, s1.y, 5);     // recombination + bremsstrahlung
		const double neu = PSG_LIN(v0.w, s0.w, 3) + PSG_LIN(v1.x, s1.x, 4);     // excitation + ionisation
		const double chi = PSG_LIN(v1.z, s1.z, 6);                           // Compton
		const double L = __fma_rn(cx.nH, __fma_rn(neu, xHI, ion * xHII), chi);
		dx[1] = __fma_rn(-cx.hpt * ye, L, cx.heat);
	}
#undef PSG_LIN
}

// Adaptive Dormand-Prince 5(4) over s in [0,1]. LSODA runs the reference at
// rtol 1e-4 (solve.c:151-152); 1e-6 here. The state of one integration is a
// DPState; dp_init() evaluates the first derivative and picks the first step
// (about a 1% change of each component, components near zero measured
// against atol/rtol), dp_step() attempts one step.
struct DPState {
	double x[2], k1[2];
	double rec, krec;   // REC: yGrecHII gained so far, and its derivative at x
	double t, h;
	float hnext;     // proposal for a step beyond s = 1 (the interval end truncates h)
	int steps;
};

#define DP_RTOL 1e-6
#define DP_ATOL0 1e-10
#define DP_ATOL1_REL 1e-8

// First step from the derivative S.k1 = f(S.x), already evaluated.
__device__ __forceinline__ void dp_init_k1(DPState &S) {
	S.t = 0.0;
	S.steps = 0;
	double h = 1.0;
	const double atol1 = DP_ATOL1_REL * fabs(S.x[1]) + 1e-300;
	for (int i = 0; i < 2; i++) {
		const double scale = fabs(S.x[i]) + (i == 0 ? DP_ATOL0 : atol1) / DP_RTOL;
		const double f = fabs(S.k1[i]);
		if (f > 0.0) h = fmin(h, 0.01 * scale / f);
	}
	S.h = fmax(h, 1e-8);
	S.hnext = 0.0f;
}

template <bool REC = false>
__device__ __forceinline__ void dp_init(const PhysParams &P, const RhsCtx &cx, DPState &S) {
	S.rec = 0.0;
	rhs<REC, true>(P, cx, S.x, S.k1, &S.krec);
	S.t = 0.0;
	S.steps = 0;
	double h = 1.0;
	const double atol1 = DP_ATOL1_REL * fabs(S.x[1]) + 1e-300;
	for (int i = 0; i < 2; i++) {
		const double scale = fabs(S.x[i]) + (i == 0 ? DP_ATOL0 : atol1) / DP_RTOL;
		const double f = fabs(S.k1[i]);
		if (f > 0.0) h = fmin(h, 0.01 * scale / f);
	}
	S.h = fmax(h, 1e-8);
	S.hnext = 0.0f;
}

// One attempted step; returns true once s = 1 is reached.
template <bool REC = false>
__device__ __forceinline__ bool dp_step(const PhysParams &P, const RhsCtx &cx, DPState &S, double atol1) {
	const double a21 = 1. / 5, a31 = 3. / 40, a32 = 9. / 40, a41 = 44. / 45, a42 = -56. / 15, a43 = 32. / 9;
	const double a51 = 19372. / 6561, a52 = -25360. / 2187, a53 = 64448. / 6561, a54 = -212. / 729;
	const double a61 = 9017. / 3168, a62 = -355. / 33, a63 = 46732. / 5247, a64 = 49. / 176, a65 = -5103. / 18656;
	const double b1 = 35. / 384, b3 = 500. / 1113, b4 = 125. / 192, b5 = -2187. / 6784, b6 = 11. / 84;
	const double e1 = 71. / 57600, e3 = -71. / 16695, e4 = 71. / 1920, e5 = -17253. / 339200, e6 = 22. / 525, e7 = -1. / 40;
	double h = S.h;
	const bool cut = S.t + h > 1.0;
	if (cut) h = 1.0 - S.t;
	double k2[2], k3[2], k4[2], k5[2], k6[2], k7[2], y[2], yn[2];
	double r2 = 0.0, r3 = 0.0, r4 = 0.0, r5 = 0.0, r6 = 0.0, r7 = 0.0;
	const double *x = S.x, *k1 = S.k1;
#define F __fma_rn
	for (int i = 0; i < 2; i++) y[i] = F(h, a21 * k1[i], x[i]);
	rhs<REC, true>(P, cx, y, k2, &r2);
	for (int i = 0; i < 2; i++) y[i] = F(h, F(a32, k2[i], a31 * k1[i]), x[i]);
	rhs<REC, true>(P, cx, y, k3, &r3);
	for (int i = 0; i < 2; i++) y[i] = F(h, F(a43, k3[i], F(a42, k2[i], a41 * k1[i])), x[i]);
	rhs<REC, true>(P, cx, y, k4, &r4);
	for (int i = 0; i < 2; i++) y[i] = F(h, F(a54, k4[i], F(a53, k3[i], F(a52, k2[i], a51 * k1[i]))), x[i]);
	rhs<REC, true>(P, cx, y, k5, &r5);
	for (int i = 0; i < 2; i++)
		y[i] = F(h, F(a65, k5[i], F(a64, k4[i], F(a63, k3[i], F(a62, k2[i], a61 * k1[i])))), x[i]);
	rhs<REC, true>(P, cx, y, k6, &r6);
	for (int i = 0; i < 2; i++) yn[i] = F(h, F(b6, k6[i], F(b5, k5[i], F(b4, k4[i], F(b3, k3[i], b1 * k1[i])))), x[i]);
	rhs<REC, true>(P, cx, yn, k7, &r7);
	double err = 0.0;
	for (int i = 0; i < 2; i++) {
		const double e = h * F(e7, k7[i], F(e6, k6[i], F(e5, k5[i], F(e4, k4[i], F(e3, k3[i], e1 * k1[i])))));
		const double sc = (i == 0 ? DP_ATOL0 : atol1) + DP_RTOL * fmax(fabs(x[i]), fabs(yn[i]));
		err += (e / sc) * (e / sc);
	}
#undef F
	// step-size control needs no double precision
	const float errf = sqrtf((float)(0.5 * err));
	if (errf <= 1.0f) {
		S.t += h;
		S.x[0] = yn[0]; S.x[1] = yn[1];
		S.k1[0] = k7[0]; S.k1[1] = k7[1];
		if (REC) {
			S.rec = __fma_rn(h, __fma_rn(b6, r6, __fma_rn(b5, r5, __fma_rn(b4, r4, __fma_rn(b3, r3, b1 * S.krec)))), S.rec);
			S.krec = r7;
		}
	}
	const float fac = errf > 0.0f ? fminf(5.0f, fmaxf(0.2f, 0.9f * __powf(errf, -0.2f))) : 5.0f;
	S.hnext = (cut && errf <= 1.0f) ? fmaxf((float)S.h, (float)h * fac) : (float)h * fac;
	S.h = fmax(h * (double)fac, 1e-14);
	S.steps++;
	return S.t >= 1.0;
}

// Stiff finish: particles whose cooling time is far below the step make the
// explicit method crawl. After DP_SWITCH steps such a particle continues
// with a Rosenbrock method (the L-stable second-order W-method with
// third-order error estimate of Shampine & Reichelt's ode23s), Jacobian by
// finite differences, rtol RB_RTOL.
#define DP_SWITCH 32
#define RB_RTOL 1e-5

// With REC, *rec accumulates yGrecHII: the third component of the augmented
// system, whose Jacobian column is zero, so W's last row only adds
// h*d*(J20*k0 + J21*k1) to its stage values; it stays out of the error norm.
template <bool REC = false>
__device__ inline bool rosenbrock(const PhysParams &P, const RhsCtx &cx, double x[2], double t, double h,
		int max_steps, double *rec = nullptr) {
	const double d = 1.0 / (2.0 + 1.4142135623730951), e32 = 6.0 + 1.4142135623730951;
	const double atol[2] = {DP_ATOL0, DP_ATOL1_REL * fabs(x[1]) + 1e-300};
	double F0[2], R0 = 0.0;
	rhs<REC>(P, cx, x, F0, &R0);
	h = fmin(fmax(h, 1e-10), 1.0);
	for (int it = 0; it < max_steps; it++) {
		if (t >= 1.0) return true;
		if (t + h > 1.0) h = 1.0 - t;
		// Jacobian by forward differences
		double J[2][2], JR[2] = {0.0, 0.0};
		for (int j = 0; j < 2; j++) {
			const double del = 1e-7 * fmax(fabs(x[j]), atol[j] / RB_RTOL);
			double y[2] = {x[0], x[1]}, Fj[2], Rj = 0.0;
			y[j] += del;
			rhs<REC>(P, cx, y, Fj, &Rj);
			J[0][j] = (Fj[0] - F0[0]) / del;
			J[1][j] = (Fj[1] - F0[1]) / del;
			if (REC) JR[j] = (Rj - R0) / del;
		}
		const double a00 = 1.0 - h * d * J[0][0], a01 = -h * d * J[0][1];
		const double a10 = -h * d * J[1][0], a11 = 1.0 - h * d * J[1][1];
		const double det = a00 * a11 - a01 * a10;
		auto solve = [&](const double b[2], double out[2]) {
			out[0] = (a11 * b[0] - a01 * b[1]) / det;
			out[1] = (a00 * b[1] - a10 * b[0]) / det;
		};
		double k1[2], k2[2], k3[2], F1[2], F2[2], y[2], yn[2], b[2], R1 = 0.0, R2 = 0.0;
		solve(F0, k1);
		const double kr1 = REC ? R0 + h * d * (JR[0] * k1[0] + JR[1] * k1[1]) : 0.0;
		y[0] = x[0] + 0.5 * h * k1[0];
		y[1] = x[1] + 0.5 * h * k1[1];
		rhs<REC>(P, cx, y, F1, &R1);
		b[0] = F1[0] - k1[0];
		b[1] = F1[1] - k1[1];
		solve(b, k2);
		const double kr2 = REC ? (R1 - kr1) + h * d * (JR[0] * k2[0] + JR[1] * k2[1]) + kr1 : 0.0;
		k2[0] += k1[0];
		k2[1] += k1[1];
		yn[0] = x[0] + h * k2[0];
		yn[1] = x[1] + h * k2[1];
		rhs<REC>(P, cx, yn, F2, &R2);
		b[0] = F2[0] - e32 * (k2[0] - F1[0]) - 2.0 * (k1[0] - F0[0]);
		b[1] = F2[1] - e32 * (k2[1] - F1[1]) - 2.0 * (k1[1] - F0[1]);
		solve(b, k3);
		double err = 0.0;
		for (int i = 0; i < 2; i++) {
			const double e = h / 6.0 * (k1[i] - 2.0 * k2[i] + k3[i]);
			const double sc = atol[i] + RB_RTOL * fmax(fabs(x[i]), fabs(yn[i]));
			err += (e / sc) * (e / sc);
		}
		err = sqrt(0.5 * err);
		if (err <= 1.0 && isfinite(err)) {
			t += h;
			x[0] = yn[0];
			x[1] = yn[1];
			F0[0] = F2[0];
			F0[1] = F2[1];
			if (REC) {
				*rec += h * kr2;
				R0 = R2;
			}
		}
		const float fac = (err > 0.0 && isfinite(err))
				? fminf(5.0f, fmaxf(0.2f, 0.9f * __powf((float)err, -1.0f / 3.0f))) : (isfinite(err) ? 5.0f : 0.2f);
		h = fmax(h * (double)fac, 1e-14);
	}
	return t >= 1.0;
}

// Whole integration on one thread; returns false if the step limit is
// reached. With REC, *rec receives the yGrecHII gained.
template <bool REC = false>
__device__ inline bool dopri(const PhysParams &P, const RhsCtx &cx, double x[2], int max_steps,
		double *rec = nullptr) {
	DPState S;
	S.x[0] = x[0];
	S.x[1] = x[1];
	const double atol1 = DP_ATOL1_REL * fabs(x[1]) + 1e-300;
	dp_init<REC>(P, cx, S);
	bool done = false;
	while (!done && S.steps < DP_SWITCH) done = dp_step<REC>(P, cx, S, atol1);
	x[0] = S.x[0];
	x[1] = S.x[1];
	if (REC) *rec = S.rec;
	if (done) return true;
	return rosenbrock<REC>(P, cx, x, S.t, S.h, max_steps, rec);
}

// step_evolve_euler() solve.c:225-316, hydrogen only: nsteps explicit Euler
// steps of the normalised system, the internal step a 200th of the shorter
// of the recombination and ionisation times at the start (rates of
// FETCH_VARS, solve.c:42-73), at most 10000 steps; the walk stops one step
// after lambdaH leaves [0, 1] and reports the unused fraction of the step
// (step_remain = 1 - (float)k / nsteps). Returns PSG_ST_* bits.
// With REC, *rec receives the yGrecHII gained (solve.c:256-300, x[3]).
template <bool REC = false>
__device__ inline uint32_t euler_step(const PhysParams &P, const RhsCtx &cx, double x[2], double &step_remain,
		int &refined, double *rec = nullptr) {
	const double ye = (1.0 - x[0]) + P.he_e + cx.yeMET;
	const double T = P.isothermal ? cx.T : ieye2T(P, x[1], ye);
	const RateAt R = rates_at(P, log10(T));
	const double alphaA = R(PSG_AR_HII_RC_A) * cx.nH;
	const double gamma = R(PSG_AR_HI_CI) * cx.nH;
	double internal = fmin(1.0 / alphaA, 1.0 / gamma) / 200.0;
	internal = fmin(internal, cx.time);
	int nsteps = (int)(cx.time / internal);
	if (nsteps > 10000) nsteps = 10000;
	if (nsteps < 1) nsteps = 1;
	const double h = 1.0 / nsteps;
	refined = nsteps > 1;
	uint32_t st = 0;
	int k;
	double acc = 0.0;
	for (k = 0; k < nsteps; k++) {
		double dx[2], r = 0.0;
		rhs<REC>(P, cx, x, dx, &r);
		if (!(x[1] + dx[1] >= 0.0)) st |= PSG_ST_IE_NEG;      // function()'s check, solve.c:137-139
		x[0] += dx[0] * h;
		x[1] += dx[1] * h;
		if (REC) acc += r * h;
		if (!isfinite(x[0]) || !isfinite(x[1])) {
			st |= PSG_ST_NAN;
			k++;
			break;
		}
		if (x[0] < 0.0 || x[0] > 1.0) {
			k++;
			break;
		}
	}
	step_remain = 1.0 - (double)((float)k / (float)nsteps);
	if (REC) *rec = acc;
	return st;
}

// Isothermal step only (the closed form), for the kernels specialised on
// it. Not on the spot, *grec (if not NULL) receives the yGrecHII gained.
__device__ inline uint32_t solve_step_iso(const PhysParams &P, double &lambdaH, double yeMET, double g,
		double time, double nH, double T, double *grec = nullptr) {
	const RateAt R = rates_at(P, log10(T));
	const double gamma = R(PSG_AR_HI_CI) * nH;
	const double alpha = R(P.on_the_spot ? PSG_AR_HII_RC_B : PSG_AR_HII_RC_A) * nH;
	const double m = yeMET + P.he_e;
	const double a = time * (alpha + gamma);
	const double b = time * (alpha + (alpha + gamma) * (1.0 + m));
	const double q = time * (gamma * (1.0 + m) + alpha * m);
	const double c = time * alpha * (1.0 + m) - g;
	const double lam0 = lambdaH;
	if (grec && !P.on_the_spot) {
		double I1 = 0.0;
		lambdaH = riccati_step(lam0, a, b, q, c, g, &I1);
		const double alpha_ab = fdim(alpha, R(PSG_AR_HII_RC_B) * nH);
		*grec = riccati_rec(lam0, lambdaH, I1, a, b, c, m, time * alpha_ab,
				alpha + gamma > 0.0 ? alpha_ab / (alpha + gamma) : 0.0);
	} else {
		lambdaH = riccati_step(lam0, a, b, q, c, g);
	}
	uint32_t st = isfinite(lambdaH) ? 0u : PSG_ST_NAN;
	if (grec && !isfinite(*grec)) st |= PSG_ST_NAN;
	lambdaH = fmin(1.0, fmax(0.0, lambdaH));
	return st;
}

// One particle step. lambdaH is clamped to [0,1] as solve.c:208 does. Not
// on the spot, *grec (if not NULL) receives the yGrecHII gained. Returns a
// PSG_ST_* bit on trouble, 0 otherwise.
__device__ inline uint32_t solve_step(const PhysParams &P, double &lambdaH, double &ie, double yeMET,
		double g, double heat, double time, double nH, double T, double *grec = nullptr) {
	uint32_t st = 0;
	if (P.isothermal) {
		st = solve_step_iso(P, lambdaH, yeMET, g, time, nH, T, grec);
	} else {
		RhsCtx cx = make_rhs_ctx(P, yeMET, g, heat, time, nH, T);
		double x[2] = {lambdaH, ie};
		double r = 0.0;
		const bool ok = (grec && !P.on_the_spot) ? dopri<true>(P, cx, x, 200000, &r) : dopri<false>(P, cx, x, 200000);
		if (!ok) st |= PSG_ST_SOLVER;
		if (grec) *grec = r;
		lambdaH = x[0];
		ie = x[1];
		if (!(ie >= 0.0)) st |= PSG_ST_IE_NEG;
	}
	if (!isfinite(lambdaH) || !isfinite(ie)) st |= PSG_ST_NAN;
	lambdaH = fmin(1.0, fmax(0.0, lambdaH));
	return st;
}
