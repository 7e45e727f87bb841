// Normalised associated Legendre functions and multiple-angle trigonometry, host and device.
#pragma once
#include "common.cuh"
#include "ref_tables.h"

namespace agb {

/** Normalised associated Legendre functions P_l^m(theta) for l = m..lmax, with their first
    and second theta-derivatives (dP, d2P may be null), as functions of tau = cos(theta) /
    (1 + sin(theta)).  Upward recurrence in l from the closed form of P_m^m, with the special
    small-sin(theta) forms of the derivatives for m = 0, 1, 2.
    Algorithm of math::sphHarmArray / legendrePmm, reference src/math_sphharm.cpp:22-132. */
AGB_HD void legendreArray(int lmax, int m, double tau, double* P, double* dP, double* d2P)
{
    if(lmax == 0) {
        P[0] = 0.5 / SQRT_PI;
        if(dP)  dP[0] = 0;
        if(d2P) d2P[0] = 0;
        return;
    }
    const double ct = 2 * tau / (1 + tau * tau);          // cos(theta)
    const double st = (1 - tau * tau) / (1 + tau * tau);  // sin(theta)
    // P_m^m = (-1)^m (2m-1)!! sin^m(theta), normalised by sqrt((2m+1) / (4 pi (2m)!));
    // the normalisations for m <= 16 come from the reference's 16-digit table
    double prefact, coef;
    if(m <= PMM_TABLE_MAX) {
#ifdef __CUDA_ARCH__
        prefact = PMM_NORM_DEV[m];
        coef = PMM_COEF_DEV[m];
#else
        prefact = PMM_NORM[m];
        coef = PMM_COEF[m];
#endif
    } else {
        double f = 1, df = 1;
        for(int k = 2; k <= 2 * m; k++) f *= k;
        for(int k = 2 * m - 1; k > 1; k -= 2) df *= k;
        prefact = 0.5 / SQRT_PI * sqrt((2 * m + 1) / f);
        coef = prefact * df * (m % 2 == 1 ? -1 : 1);
    }
    if(m == 0) {
        P[0] = prefact;
        if(dP)  dP[0] = 0;
        if(d2P) d2P[0] = 0;
    } else if(m == 1) {
        P[0] = -st * prefact;
        if(dP)  dP[0] = -ct * prefact;
        if(d2P) d2P[0] = st * prefact;
    } else {
        // sin^(m-2) by binary exponentiation (same product order as the reference's math::pow)
        double sinm2 = 1, base = st;
        for(int e = m - 2; ; ) {
            if(e % 2) sinm2 *= base;
            e >>= 1;
            base *= base;
            if(!e) break;
        }
        P[0] = coef * sinm2 * (st * st);
        if(dP)  dP[0] = m * coef * sinm2 * st * ct;
        if(d2P) d2P[0] = m * coef * sinm2 * (m * (ct * ct) - 1);
    }
    if(lmax == m)
        return;
    double Plm1 = P[0] / prefact, Plm = ct * (2 * m + 1) * Plm1, Plm2 = 0;
    double d2Plm1 = st, d2Plm2 = 0, d2Plm = 12 * ct * st;   // special m == 1 second derivatives
    const double EPS = 1e-8;                                  // small-sin(theta) threshold
    for(int l = m + 1; l <= lmax; l++) {
        const int i = l - m;
        if(l > m + 1)
            Plm = (ct * (2 * l - 1) * Plm1 - (l + m - 1) * Plm2) / (l - m);
        prefact *= sqrt((2 * l + 1.) / (2 * l - 1.) * (l - m) / (l + m));
        P[i] = Plm * prefact;
        if(dP) {
            double dPlm = 0;
            if(st >= EPS || (m > 2 && st > 0))
                dPlm = (l * ct * Plm - (l + m) * Plm1) / st;
            else if(m == 0)
                dPlm = -l * (l + 1) / 2 * st * (ct > 0 || l % 2 == 1 ? 1 : -1);
            else if(m == 1)
                dPlm = -l * (l + 1) / 2 * (ct > 0 || l % 2 == 0 ? 1 : -1);
            else if(m == 2)
                dPlm = l * (l + 1) * (l + 2) * (l - 1) / 4 * st * (ct > 0 || l % 2 == 1 ? 1 : -1);
            dP[i] = prefact * dPlm;
        }
        if(d2P) {
            if(st >= EPS || (m > 2 && st > 0))
                d2P[i] = ct * dP[i] / (-st) - (l * (l + 1) - pow2(m / st)) * P[i];
            else if(m == 0)
                d2P[i] = -l * (l + 1) / 2 * prefact * (ct > 0 || l % 2 == 0 ? 1 : -1);
            else if(m == 1) {
                if(l > m + 1) {
                    const double twodPlm1 = -l * (l - 1) * (ct > 0 || l % 2 == 1 ? 1 : -1);
                    d2Plm = ((2 * l - 1) * (ct * (d2Plm1 - Plm1) - st * twodPlm1) - l * d2Plm2) / (l - 1);
                }
                d2P[i] = prefact * d2Plm;
                d2Plm2 = d2Plm1;
                d2Plm1 = d2Plm;
            } else if(m == 2)
                d2P[i] = l * (l + 1) * (l + 2) * (l - 1) / 4 * prefact * (ct > 0 || l % 2 == 0 ? 1 : -1);
            else
                d2P[i] = 0;
        }
        Plm2 = Plm1;
        Plm1 = Plm;
    }
}

/** cos(k phi) (out[k-1]) and, if needSine, sin(k phi) (out[m+k-1]) for k = 1..m, by the
    rotation recurrence with alpha = 2 sin^2(phi/2), beta = sin(phi) (Numerical Recipes 3rd ed.
    sec. 5.4); the reference's trigMultiAngle, src/math_sphharm.cpp:134-154. */
AGB_HD void trigMultiAngle(double phi, int m, bool needSine, double* out)
{
    if(m < 1) return;
    double s1, c1, sh, ch;
    sincos(phi, &s1, &c1);
    sincos(0.5 * phi, &sh, &ch);
    const double alpha = 2 * sh * sh, beta = s1;
    double cprev = 1, sprev = 0;
    for(int k = 0; k < m; k++) {
        const double c = cprev - (alpha * cprev + beta * sprev);
        const double s = sprev - (alpha * sprev - beta * cprev);
        out[k] = c;
        if(needSine) out[k + m] = s;
        cprev = c;
        sprev = s;
    }
}

}  // namespace agb
