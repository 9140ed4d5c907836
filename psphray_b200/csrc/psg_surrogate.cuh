// Inputs and outputs of the chemistry surrogate, shared by the update log
// (training data), the training set-up and the inference kernel.
//
// The network sees one particle's step (not isothermal) through five
// inputs, all base-10 logarithms:
//   f0 = nH * time            the recombination column of the step (the
//                             step length varies per particle: nH alone
//                             cannot set the update)
//   f1 = T at the start
//   f2 = logit(lambdaH) = log(lambdaH) - log(1 - lambdaH)   (both the
//                             neutral and the ionised fraction, in one)
//   f3 = g                    photons absorbed per H over the step
//   f4 = heat / ie            photo-heating over the step, relative
// and predicts
//   y0 = logit(lambdaH') - logit(lambdaH),  y1 = log T' - log T.
#pragma once

#include "psg_solve.cuh"

#define PSG_SURR_NFEAT 5
#define PSG_SURR_LAM_MIN 1e-12

__device__ __forceinline__ double surr_logit(double lam) {
	lam = fmin(fmax(lam, PSG_SURR_LAM_MIN), 1.0 - PSG_SURR_LAM_MIN);
	return log10(lam) - log10(1.0 - lam);
}
__device__ __forceinline__ double surr_unlogit(double u) {
	// lambda = 1 / (1 + 10^-u)
	return 1.0 / (1.0 + exp10(-u));
}

__device__ __forceinline__ void surr_features(const RhsCtx &cx, double lam0, double ie0, float f[PSG_SURR_NFEAT]) {
	f[0] = (float)log10(fmax(cx.nH * cx.time, 1e-300));
	f[1] = (float)log10(fmax(cx.T, 1e-300));
	f[2] = (float)surr_logit(lam0);
	// below 1e-16 photons (or heat) per atom a step is no longer driven: a
	// floor keeps the inputs of undriven particles next to the others
	f[3] = (float)log10(fmax(cx.g, 1e-16));
	f[4] = (float)log10(fmax(cx.heat / fmax(ie0, 1e-300), 1e-16));
}
