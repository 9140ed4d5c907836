/* C restatement of the reference's src/verner.F90 (three photo-ionisation
 * cross sections, single-precision Fortran `real` functions). No Fortran
 * compiler exists in this image, so the reference's atomic-rate.c is linked
 * against these instead. Fortran mixed-mode rules are followed: a `real`
 * operand meeting a `d0` literal is promoted to double and the result is
 * rounded back to float on assignment.
 *
 *   verner_hi_photo_cs_      verner.F90:7-33   (Verner et al. 1996 HI fit)
 *   osterbrok_hei_photo_cs_  verner.F90:37-51  (Osterbrock HeI)
 *   osterbrok_heii_photo_cs_ verner.F90:55-65  (Osterbrock HeII)
 *
 * This file is test infrastructure for the oracle build only. */
#include <math.h>

float verner_hi_photo_cs_(const float *Ry) {
	const float E0 = 4.298e-1f;     /* real, parameter :: E0 = 4.298d-1 */
	const float sig0 = 5.475e4f;
	const float ya = 3.288e1f;
	const float P = 2.963f;
	if (*Ry < 0.5f) return 0.0f;
	const float eV = (float)((double)*Ry * 13.6);      /* Ry * 13.6d0 */
	const float x = eV / E0;
	const float y = x;
	const float xm1 = x - 1.0f;
	const float a = sig0 * (xm1 * xm1);                /* sig0 * (x-1)**2 */
	const double e = 0.5 * (double)P - 5.5;            /* 0.5d0*P - 5.5d0 */
	const double b = (double)a * pow((double)y, e);
	const float c = powf(1.0f + sqrtf(y / ya), -P);
	float sigma = (float)(b * (double)c);
	sigma = (float)((double)sigma * 1.0e-18);
	if (sigma < 0.0f) sigma = 0.0f;
	return sigma;
}

float osterbrok_hei_photo_cs_(const float *Ry) {
	const float nu = 24.587f;
	if (2.0f * *Ry * 13.6f < nu) return 0.0f;
	const float sf = *Ry * 13.6f / nu;
	return 7.2e-18f * (1.66f * powf(sf, -2.05f) + 0.66f * powf(sf, -3.05f));
}

float osterbrok_heii_photo_cs_(const float *Ry) {
	const float nu = 54.416f;
	if (2.0f * *Ry * 13.6f < nu) return 0.0f;
	const float s = *Ry * 13.6f / nu;
	return 1.58e-18f * (1.0f / (s * s * s));
}
