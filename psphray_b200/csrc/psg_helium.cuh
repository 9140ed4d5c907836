// Helium and secondary ionisation on the device (psphray.HOnly = false,
// psphray.secondaryIonization): the cross sections of the three species,
// the secondary-ionisation table lookup, and the update of one particle
// over the four variables (lambdaH, lambdaHeI, lambdaHeII, ie) of
// function() solve.c:76-141.
//
// The isothermal closed form does not apply once helium's electrons enter
// ye, so every helium update is integrated: Dormand-Prince 5(4) (rtol 1e-6)
// for up to HE_SWITCH steps, then a Rosenbrock W-method (ode23s, rtol 1e-5,
// LU with partial pivoting of the 4x4 W) for particles stiffer than that;
// or, with the explicit build, step_evolve_euler() solve.c:225-316.
#pragma once

#include "psg_solve.cuh"

// xs_get() atomic-rate.c:126-131 for species s (0 HI, 1 HeI, 2 HeII)
__device__ __forceinline__ double xs_get_s(const PhysParams &P, int s, double freq) {
	const double cut = s == 0 ? P.xs_cut_HI : (s == 1 ? P.xs_cut_HeI : P.xs_cut_HeII);
	if (freq < cut) return 0.0;
	return tab_get(P.xs_nrows, P.xs_min, P.xs_step_inv, P.xs, P.xs + (size_t)(1 + s) * P.xs_nrows, freq);
}

// secion_get() secion.c:100-103 = tabfun2_get() tabfun.c:173-222 on column
// col (0 PhiHI, 1 PhiHeI, 2 Eh): clamped rows or columns interpolate along
// the other axis, inside the table bilinear; the grid values are
// min + i*step as tabfun2 stores them.
__device__ inline double secion_get(const PhysParams &P, int col, double E, double y) {
	const int n1 = PSG_SECION_NE, n2 = PSG_SECION_NX;
	const double *d = P.si + (size_t)col * n1 * n2;
	const int xind = (int)((E - P.si_min1) * P.si_step1_inv);
	const int yind = (int)((y - P.si_min2) * P.si_step2_inv);
	int lo = -1;
	if (xind < 0) lo = 0;
	if (xind >= n1 - 1) lo = (n1 - 1) * n2;
	if (lo != -1) {
		if (yind < 0) return d[lo];
		if (yind >= n2 - 1) return d[lo + n2 - 1];
		const double left = P.si_min2 + yind * P.si_step2, right = P.si_min2 + (yind + 1) * P.si_step2;
		return ((right - y) * d[lo + yind] + (y - left) * d[lo + yind + 1]) * P.si_step2_inv;
	}
	int lin = -1;
	if (yind < 0) lin = 0;
	if (yind >= n2 - 1) lin = n2 - 1;
	if (lin != -1) {
		const double left = P.si_min1 + xind * P.si_step1, right = P.si_min1 + (xind + 1) * P.si_step1;
		return ((right - E) * d[(size_t)xind * n2 + lin] + (E - left) * d[(size_t)(xind + 1) * n2 + lin]) *
				P.si_step1_inv;
	}
	const double x1 = P.si_min1 + xind * P.si_step1, x2 = P.si_min1 + (xind + 1) * P.si_step1;
	const double y1 = P.si_min2 + yind * P.si_step2, y2 = P.si_min2 + (yind + 1) * P.si_step2;
	const double fac = P.si_step1_inv * P.si_step2_inv;
	const double f11 = d[(size_t)xind * n2 + yind], f12 = d[(size_t)xind * n2 + yind + 1];
	const double f21 = d[(size_t)(xind + 1) * n2 + yind], f22 = d[(size_t)(xind + 1) * n2 + yind + 1];
	return fac * (f11 * (x2 - E) * (y2 - y) + f21 * (E - x1) * (y2 - y) + f12 * (x2 - E) * (y - y1) +
			f22 * (E - x1) * (y - y1));
}

// lambda_to_ye() psystem.h:134-138 (without yeMET)
__device__ __forceinline__ double ye_he(const PhysParams &P, double lamH, double l1, double l2) {
	return (1.0 - lamH) + P.hemf / P.hmf * 0.25 * (l2 + 2 * (1.0 - l2 - l1));
}

// The rate columns at one log T from the FP32 (value, slope) rows (each
// column scaled by its largest magnitude): the two-point line of
// tabfun_get() tabfun.c:38-58 written as value + slope * offset; a column
// is one 8-byte load.
struct RateRow {
	const float2 *row;
	double du;
	const double *scale;
	__device__ __forceinline__ double operator()(int c) const {
		const float2 vs = row[c];
		return __fma_rn((double)vs.y, du, (double)vs.x) * scale[c];
	}
};

__device__ __forceinline__ RateRow rate_row(const PhysParams &P, double logT) {
	long long idx = (long long)((logT - P.ar_min) * P.ar_step_inv);
	RateRow R;
	if (idx < 0) {
		idx = 0;
		R.du = 0.0;
	} else if (idx >= P.ar_nrows - 1) {
		idx = P.ar_nrows - 1;
		R.du = 0.0;
	} else {
		R.du = logT - __fma_rn((double)idx, P.ar_step, P.ar_min);
	}
	R.row = P.ar_all + 16 * idx;
	R.scale = P.ar_all_scale;
	return R;
}

// One helium step: the Step fields the right-hand side reads.
struct HeStep {
	double yeMET, gHI, gHeI, gHeII, heat, time, nH, T;
};

// function() solve.c:76-141 with helium (the rates of FETCH_VARS
// solve.c:42-73); x = (lambdaH, lambdaHeI, lambdaHeII, ie), the derivative
// per unit normalised time. On the spot (case B) the helium equations use
// x_HI where solve.c:94-95 writes it; not on the spot (case A) rec[3]
// receives the recombination photons' rates d(yGrecHII, yGrecHeII,
// yGrecHeIII)/ds of solve.c:84-91.
__device__ inline void rhs_he(const PhysParams &P, const HeStep &s, const double x[4], double dx[4],
		double *rec = nullptr) {
	const double xHI = x[0], xHII = 1.0 - x[0], xHeII = x[2];
	const double xHeIII = 1.0 - x[2] - x[1];
	const double ye = (xHII + P.hemf / P.hmf * 0.25 * (xHeII + 2 * xHeIII)) + s.yeMET;
	const double T = P.isothermal ? s.T : ieye2T(P, x[3], ye);
	const RateRow R = rate_row(P, log10(T));
	const double nH = s.nH, t = s.time;
	const double gamma_HI = R(PSG_AR_HI_CI) * nH;
	const double gamma_HeI = R(PSG_AR_HEI_CI) * nH;
	const double gamma_HeII = R(PSG_AR_HEII_CI) * nH;
	const double aHII_B = R(PSG_AR_HII_RC_B) * nH, aHeII_B = R(PSG_AR_HEII_RC_B) * nH;
	const double aHeIII_B = R(PSG_AR_HEIII_RC_B) * nH;
	if (P.on_the_spot) {
		dx[0] = (-s.gHI / t + (-gamma_HI * ye * xHI + aHII_B * ye * xHII)) * t;
		dx[1] = (-s.gHeI / t + (-gamma_HeI * ye * xHI + aHeII_B * ye * xHeII)) * t;
		dx[2] = (-s.gHeII / t + (-gamma_HeII * ye * xHI - aHeII_B * ye * xHeII + aHeIII_B * ye * xHeIII)) * t;
	} else {
		const double xHeI = x[1];
		const double aHII_A = R(PSG_AR_HII_RC_A) * nH, aHeII_A = R(PSG_AR_HEII_RC_A) * nH;
		const double aHeIII_A = R(PSG_AR_HEIII_RC_A) * nH;
		dx[0] = (-s.gHI / t + (-gamma_HI * ye * xHI + aHII_A * ye * xHII)) * t;
		dx[1] = (-s.gHeI / t + (-gamma_HeI * ye * xHeI + aHeII_A * ye * xHeII)) * t;
		dx[2] = (-s.gHeII / t + (-gamma_HeII * ye * xHeII - aHeII_A * ye * xHeII + aHeIII_A * ye * xHeIII)) * t;
		if (rec) {
			rec[0] = fdim(aHII_A, aHII_B) * ye * xHII * t;
			rec[1] = fdim(aHeII_A, aHeII_B) * ye * xHeII * t;
			rec[2] = fdim(aHeIII_A, aHeIII_B) * ye * xHeIII * t;
		}
	}
	if (P.isothermal || P.adiabatic) {
		dx[3] = 0.0;
	} else {
		const double eta = R(P.on_the_spot ? PSG_AR_HII_RCC_B : PSG_AR_HII_RCC_A) * nH;
		const double psi = R(PSG_AR_HI_CEC) * nH, zeta = R(PSG_AR_HI_CIC) * nH;
		const double beta = R(PSG_AR_E_BREMC) * nH, chi = R(PSG_AR_E_COMPC);
		const double L = P.H_PER_MASS * ((zeta + psi) * ye * xHI + (eta * ye * xHII) + beta * ye * xHII + chi * ye);
		dx[3] = (s.heat / t - L) * t;
	}
}

#define HE_SWITCH 32

__device__ __forceinline__ double he_err_norm(const double e[4], const double x[4], const double y[4], double atol3,
		double rtol) {
	double err = 0.0;
	for (int i = 0; i < 4; i++) {
		const double sc = (i < 3 ? DP_ATOL0 : atol3) + rtol * fmax(fabs(x[i]), fabs(y[i]));
		err += (e[i] / sc) * (e[i] / sc);
	}
	return sqrt(0.25 * err);
}

// Rosenbrock ode23s over the four variables from (t, x) with step h. With
// rec (not on the spot) the three recombination-photon counts are carried
// as extra components whose Jacobian columns are zero: W's extra rows add
// h*d*(J_r . k) to their stage values; they stay out of the error norm.
__device__ inline bool rosenbrock_he(const PhysParams &P, const HeStep &s, double x[4], double t, double h,
		int max_steps, double *rec = nullptr) {
	const double d = 1.0 / (2.0 + 1.4142135623730951), e32 = 6.0 + 1.4142135623730951;
	const double atol3 = DP_ATOL1_REL * fabs(x[3]) + 1e-300;
	double F0[4], R0[3] = {0.0, 0.0, 0.0};
	rhs_he(P, s, x, F0, rec ? R0 : nullptr);
	h = fmin(fmax(h, 1e-10), 1.0);
	for (int it = 0; it < max_steps; it++) {
		if (t >= 1.0) return true;
		if (t + h > 1.0) h = 1.0 - t;
		double W[4][4], JR[3][4];
		for (int j = 0; j < 4; j++) {
			const double del = 1e-7 * fmax(fabs(x[j]), (j < 3 ? DP_ATOL0 : atol3) / RB_RTOL);
			double y[4] = {x[0], x[1], x[2], x[3]}, Fj[4], Rj[3] = {0.0, 0.0, 0.0};
			y[j] += del;
			rhs_he(P, s, y, Fj, rec ? Rj : nullptr);
			for (int i = 0; i < 4; i++) W[i][j] = (i == j ? 1.0 : 0.0) - h * d * (Fj[i] - F0[i]) / del;
			for (int i = 0; i < 3; i++) JR[i][j] = (Rj[i] - R0[i]) / del;
		}
		// LU with partial pivoting, in place
		int piv[4];
		bool sing = false;
		for (int k = 0; k < 4; k++) {
			int m = k;
			for (int i = k + 1; i < 4; i++)
				if (fabs(W[i][k]) > fabs(W[m][k])) m = i;
			piv[k] = m;
			if (m != k)
				for (int j = 0; j < 4; j++) {
					const double tmp = W[k][j];
					W[k][j] = W[m][j];
					W[m][j] = tmp;
				}
			if (W[k][k] == 0.0) {
				sing = true;
				break;
			}
			for (int i = k + 1; i < 4; i++) {
				W[i][k] /= W[k][k];
				for (int j = k + 1; j < 4; j++) W[i][j] -= W[i][k] * W[k][j];
			}
		}
		if (sing) return false;
		auto solve = [&](const double b[4], double out[4]) {
			double v[4] = {b[0], b[1], b[2], b[3]};
			for (int k = 0; k < 4; k++) {
				const double tmp = v[k];
				v[k] = v[piv[k]];
				v[piv[k]] = tmp;
			}
			for (int i = 1; i < 4; i++)
				for (int j = 0; j < i; j++) v[i] -= W[i][j] * v[j];
			for (int i = 3; i >= 0; i--) {
				for (int j = i + 1; j < 4; j++) v[i] -= W[i][j] * v[j];
				v[i] /= W[i][i];
			}
			for (int i = 0; i < 4; i++) out[i] = v[i];
		};
		double k1[4], k2[4], k3[4], F1[4], F2[4], y[4], yn[4], b[4], e[4];
		double R1[3] = {0.0, 0.0, 0.0}, R2[3] = {0.0, 0.0, 0.0}, kr1[3], kr2[3];
		solve(F0, k1);
		for (int i = 0; i < 3; i++)
			kr1[i] = R0[i] + h * d * (JR[i][0] * k1[0] + JR[i][1] * k1[1] + JR[i][2] * k1[2] + JR[i][3] * k1[3]);
		for (int i = 0; i < 4; i++) y[i] = x[i] + 0.5 * h * k1[i];
		rhs_he(P, s, y, F1, rec ? R1 : nullptr);
		for (int i = 0; i < 4; i++) b[i] = F1[i] - k1[i];
		solve(b, k2);
		for (int i = 0; i < 3; i++)
			kr2[i] = (R1[i] - kr1[i]) + h * d * (JR[i][0] * k2[0] + JR[i][1] * k2[1] + JR[i][2] * k2[2] +
					JR[i][3] * k2[3]) + kr1[i];
		for (int i = 0; i < 4; i++) {
			k2[i] += k1[i];
			yn[i] = x[i] + h * k2[i];
		}
		rhs_he(P, s, yn, F2, rec ? R2 : nullptr);
		for (int i = 0; i < 4; i++) b[i] = F2[i] - e32 * (k2[i] - F1[i]) - 2.0 * (k1[i] - F0[i]);
		solve(b, k3);
		for (int i = 0; i < 4; i++) e[i] = h / 6.0 * (k1[i] - 2.0 * k2[i] + k3[i]);
		const double err = he_err_norm(e, x, yn, atol3, RB_RTOL);
		if (err <= 1.0 && isfinite(err)) {
			t += h;
			for (int i = 0; i < 4; i++) {
				x[i] = yn[i];
				F0[i] = F2[i];
			}
			if (rec)
				for (int i = 0; i < 3; i++) {
					rec[i] += h * kr2[i];
					R0[i] = R2[i];
				}
		}
		const double fac = (err > 0.0 && isfinite(err)) ? fmin(5.0, fmax(0.2, 0.9 * pow(err, -1.0 / 3.0)))
				: (isfinite(err) ? 5.0 : 0.2);
		h = fmax(h * fac, 1e-14);
	}
	return t >= 1.0;
}

// Up to HE_SWITCH Dormand-Prince 5(4) steps over the four variables from
// s = 0; returns true once s = 1 is reached, else leaves the time reached
// and the next step size in *t_out, *h_out. With rec (not on the spot),
// rec[3] accumulates the recombination photons as a quadrature over the
// same stages.
template <bool REC>
__device__ inline bool dopri_he_explicit(const PhysParams &P, const HeStep &s, double x[4], double *rec,
		double *t_out, double *h_out) {
	const double a21 = 1. / 5, a31 = 3. / 40, a32 = 9. / 40, a41 = 44. / 45, a42 = -56. / 15, a43 = 32. / 9;
	const double a51 = 19372. / 6561, a52 = -25360. / 2187, a53 = 64448. / 6561, a54 = -212. / 729;
	const double a61 = 9017. / 3168, a62 = -355. / 33, a63 = 46732. / 5247, a64 = 49. / 176, a65 = -5103. / 18656;
	const double b1 = 35. / 384, b3 = 500. / 1113, b4 = 125. / 192, b5 = -2187. / 6784, b6 = 11. / 84;
	const double e1 = 71. / 57600, e3 = -71. / 16695, e4 = 71. / 1920, e5 = -17253. / 339200, e6 = 22. / 525,
			e7 = -1. / 40;
	const double atol3 = DP_ATOL1_REL * fabs(x[3]) + 1e-300;
	double k1[4], r1[3] = {0.0, 0.0, 0.0};
	rhs_he(P, s, x, k1, REC ? r1 : nullptr);
	double h = 1.0;
	for (int i = 0; i < 4; i++) {
		const double scale = fabs(x[i]) + (i < 3 ? DP_ATOL0 : atol3) / DP_RTOL;
		if (fabs(k1[i]) > 0.0) h = fmin(h, 0.01 * scale / fabs(k1[i]));
	}
	h = fmax(h, 1e-8);
	double t = 0.0;
	for (int it = 0; it < HE_SWITCH; it++) {
		if (t >= 1.0) return true;
		if (t + h > 1.0) h = 1.0 - t;
		double k2[4], k3[4], k4[4], k5[4], k6[4], k7[4], y[4], yn[4], e[4];
		double r2[3], r3[3], r4[3], r5[3], r6[3], r7[3];
		double *q2 = REC ? r2 : nullptr, *q3 = REC ? r3 : nullptr, *q4 = REC ? r4 : nullptr;
		double *q5 = REC ? r5 : nullptr, *q6 = REC ? r6 : nullptr, *q7 = REC ? r7 : nullptr;
		for (int i = 0; i < 4; i++) y[i] = x[i] + h * (a21 * k1[i]);
		rhs_he(P, s, y, k2, q2);
		for (int i = 0; i < 4; i++) y[i] = x[i] + h * (a31 * k1[i] + a32 * k2[i]);
		rhs_he(P, s, y, k3, q3);
		for (int i = 0; i < 4; i++) y[i] = x[i] + h * (a41 * k1[i] + a42 * k2[i] + a43 * k3[i]);
		rhs_he(P, s, y, k4, q4);
		for (int i = 0; i < 4; i++) y[i] = x[i] + h * (a51 * k1[i] + a52 * k2[i] + a53 * k3[i] + a54 * k4[i]);
		rhs_he(P, s, y, k5, q5);
		for (int i = 0; i < 4; i++)
			y[i] = x[i] + h * (a61 * k1[i] + a62 * k2[i] + a63 * k3[i] + a64 * k4[i] + a65 * k5[i]);
		rhs_he(P, s, y, k6, q6);
		for (int i = 0; i < 4; i++) yn[i] = x[i] + h * (b1 * k1[i] + b3 * k3[i] + b4 * k4[i] + b5 * k5[i] + b6 * k6[i]);
		rhs_he(P, s, yn, k7, q7);
		for (int i = 0; i < 4; i++)
			e[i] = h * (e1 * k1[i] + e3 * k3[i] + e4 * k4[i] + e5 * k5[i] + e6 * k6[i] + e7 * k7[i]);
		const double err = he_err_norm(e, x, yn, atol3, DP_RTOL);
		if (err <= 1.0) {
			t += h;
			for (int i = 0; i < 4; i++) {
				x[i] = yn[i];
				k1[i] = k7[i];
			}
			if (REC)
				for (int i = 0; i < 3; i++) {
					rec[i] += h * (b1 * r1[i] + b3 * r3[i] + b4 * r4[i] + b5 * r5[i] + b6 * r6[i]);
					r1[i] = r7[i];
				}
		}
		const double fac = err > 0.0 ? fmin(5.0, fmax(0.2, 0.9 * pow(err, -0.2))) : 5.0;
		h = fmax(h * fac, 1e-14);
	}
	*t_out = t;
	*h_out = h;
	return t >= 1.0;
}

// Dormand-Prince 5(4) over the four variables, then the Rosenbrock finish.
__device__ inline bool dopri_he(const PhysParams &P, const HeStep &s, double x[4], int max_steps,
		double *rec = nullptr) {
	double t = 0.0, h = 0.0;
	const bool done = rec ? dopri_he_explicit<true>(P, s, x, rec, &t, &h) : dopri_he_explicit<false>(P, s, x, rec, &t, &h);
	if (done) return true;
	return rosenbrock_he(P, s, x, t, h, max_steps, rec);
}

// step_evolve_euler() solve.c:225-316 with helium: the internal step a
// 200th of the shortest recombination and ionisation time at the start,
// at most 10000 steps, stopping one step after a fraction leaves [0, 1] or
// x_HeIII turns negative. Returns PSG_ST_* bits.
__device__ inline uint32_t euler_he(const PhysParams &P, const HeStep &s, double x[4], double &step_remain,
		int &refined, double *rec = nullptr) {
	const double ye = (1.0 - x[0] + P.hemf / P.hmf * 0.25 * (x[2] + 2 * (1.0 - x[2] - x[1]))) + s.yeMET;
	const double T = P.isothermal ? s.T : ieye2T(P, x[3], ye);
	const RateAt R = rates_at(P, log10(T));
	double rectime = 1.0 / (R(PSG_AR_HII_RC_A) * s.nH);
	double iontime = 1.0 / (R(PSG_AR_HI_CI) * s.nH);
	rectime = fmin(rectime, 1.0 / (R(PSG_AR_HEII_RC_A) * s.nH));
	rectime = fmin(rectime, 1.0 / (R(PSG_AR_HEIII_RC_A) * s.nH));
	iontime = fmin(iontime, 1.0 / (R(PSG_AR_HEI_CI) * s.nH));
	iontime = fmin(iontime, 1.0 / (R(PSG_AR_HEII_CI) * s.nH));
	double internal = fmin(rectime, iontime) / 200.;
	internal = fmin(internal, s.time);
	int nsteps = (int)(s.time / internal);
	if (nsteps > 10000) nsteps = 10000;
	if (nsteps < 1) nsteps = 1;
	const double h = 1.0 / nsteps;
	refined = nsteps > 1;
	uint32_t st = 0;
	int k;
	for (k = 0; k < nsteps; k++) {
		double dx[4], r[3] = {0.0, 0.0, 0.0};
		rhs_he(P, s, x, dx, rec ? r : nullptr);
		if (!(x[3] + dx[3] >= 0.0)) st |= PSG_ST_IE_NEG;
		for (int i = 0; i < 4; i++) x[i] += dx[i] * h;
		if (rec)
			for (int i = 0; i < 3; i++) rec[i] += r[i] * h;
		if (!isfinite(x[0]) || !isfinite(x[1]) || !isfinite(x[2]) || !isfinite(x[3])) {
			st |= PSG_ST_NAN;
			k++;
			break;
		}
		bool out = false;
		for (int i = 0; i < 3; i++) out |= (x[i] < 0.0 || x[i] > 1.0);
		if (out || 1.0 - x[1] - x[2] < 0.0) {
			k++;
			break;
		}
	}
	step_remain = 1.0 - (double)((float)k / (float)nsteps);
	return st;
}

// LSODA's exit clamps of the fractions (solve.c:208-210).
__device__ __forceinline__ void clamp_he(double x[4]) {
	x[0] = fmin(1., fmax(0., x[0]));
	x[1] = fmin(1., fmax(0., x[1]));
	x[2] = fmin(1. - x[1], fmax(0., x[2]));
}

// One helium step of step_evolve() (LSODA's exit clamps, solve.c:208-213):
// x = (lambdaH, lambdaHeI, lambdaHeII, ie) in and out; with rec (not on the
// spot) the three recombination-photon counts in and out. Returns PSG_ST_*
// bits.
__device__ inline uint32_t solve_step_he(const PhysParams &P, const HeStep &s, double x[4],
		double *rec = nullptr) {
	uint32_t st = 0;
	double gain[3] = {0.0, 0.0, 0.0};
	if (!dopri_he(P, s, x, 200000, rec ? gain : nullptr)) st |= PSG_ST_SOLVER;
	if (rec)
		for (int i = 0; i < 3; i++) rec[i] = fmax(0.0, rec[i] + gain[i]);
	if (!(x[3] >= 0.0)) st |= PSG_ST_IE_NEG;
	for (int i = 0; i < 4; i++)
		if (!isfinite(x[i])) st |= PSG_ST_NAN;
	x[0] = fmin(1., fmax(0., x[0]));
	x[1] = fmin(1., fmax(0., x[1]));
	x[2] = fmin(1. - x[1], fmax(0., x[2]));
	return st;
}
