// Device evaluation of the Multipole potential, its gradient and Hessian.
//
// One thread evaluates one point.  The 2-D spline tables stay resident in L2 (they are
// 0.1-1.3 MB for the benchmark potentials); each evaluation gathers the 4 corner nodes of
// one grid cell per azimuthal harmonic (4 x 9 doubles) with 16-byte loads.
#pragma once
#include "common.cuh"
#include "multipole.h"
#include "sphharm.cuh"

namespace agb {

/// gradient in (R, z, phi) and Hessian (RR, zz, phiphi, Rz, zphi, Rphi) in cylindrical coords
struct CylDerivs { double dR, dz, dphi; };
struct CylHess   { double dR2, dz2, dphi2, dRdz, dzdphi, dRdphi; };
/// derivatives in "spherical-like" coordinates (first: ln r or r, second: theta or tau, phi)
struct SphDerivs { double dr, dt, dphi; };
struct SphHess   { double dr2, dt2, dphi2, drdt, dtdphi, drdphi; };

#ifdef __CUDACC__
__device__ __forceinline__ double ldg(const double* p) { return __ldg(p); }
__device__ __forceinline__ double2 ldg2(const double* p) { return __ldg(reinterpret_cast<const double2*>(p)); }
#endif

/** Sum of the azimuthal harmonics C_m(...) cos/sin(m phi) and their phi-derivatives; C holds
    nq blocks of nm values (value, d/dr, d/dtheta, d2/dr2, d2/drdtheta, d2/dtheta2).
    Reference fourierTransformAzimuth, src/potential_multipole.cpp:666-717. */
template<int NQ>
__device__ __forceinline__ void fourierSum(const HarmIndices& ind, double phi, const double* C,
    double* val, SphDerivs* g, SphHess* h)
{
    const int mmin = ind.mmin(), nm = ind.mmax - mmin + 1;
    *val = C[-mmin];
    if(NQ >= 3) { g->dr = C[-mmin + nm]; g->dt = C[-mmin + 2 * nm]; g->dphi = 0; }
    if(NQ == 6) {
        h->dr2 = C[-mmin + 3 * nm]; h->drdt = C[-mmin + 4 * nm]; h->dt2 = C[-mmin + 5 * nm];
        h->drdphi = h->dtdphi = h->dphi2 = 0;
    }
    if(ind.mmax == 0) return;
    const bool useSine = mmin < 0 || NQ > 1;
    double trig[2 * LMAX_MAX];
    trigMultiAngle(phi, ind.mmax, useSine, trig);
    for(int mm = 0; mm < nm; mm++) {
        const int m = mm + mmin;
        if(m == 0 || ind.lmin(m) > ind.lmax) continue;
        const double tr  = m > 0 ? trig[m - 1] : trig[ind.mmax - m - 1];
        const double dtr = m > 0 ? -m * trig[ind.mmax + m - 1] : -m * trig[-m - 1];
        const double d2tr = -m * m * tr;
        *val += C[mm] * tr;
        if(NQ >= 3) {
            g->dr   += C[mm + nm] * tr;
            g->dt   += C[mm + 2 * nm] * tr;
            g->dphi += C[mm] * dtr;
        }
        if(NQ == 6) {
            h->dr2    += C[mm + 3 * nm] * tr;
            h->drdt   += C[mm + 4 * nm] * tr;
            h->dt2    += C[mm + 5 * nm] * tr;
            h->drdphi += C[mm + nm] * dtr;
            h->dtdphi += C[mm + 2 * nm] * dtr;
            h->dphi2  += C[mm] * d2tr;
        }
    }
}

/** Inverse spherical-harmonic transform of coefficients C_lm(r) and their radial derivatives
    into value/gradient/Hessian in (r-like, theta, phi).  Reference
    sphHarmTransformInverseDeriv(2), src/potential_multipole.cpp:722-821. */
template<int NQ, class Coef>
__device__ void sphHarmInverse(const HarmIndices& ind, double R, double z, double phi,
    const Coef& coef, double* val, SphDerivs* g, SphHess* h)
{
    if(ind.lmax == 2 && ind.mmin() == 0 && ind.step == 2) {
        // closed form for the {l=0}, {l=2,m=0}, {l=2,m=2} terms
        const int i00 = 0, i20 = 6, i22 = 8;
        double C[9], dC[9], d2C[9];
        coef(i00, &C[i00], &dC[i00], &d2C[i00]);
        coef(i20, &C[i20], &dC[i20], &d2C[i20]);
        if(ind.mmax == 2) coef(i22, &C[i22], &dC[i22], &d2C[i22]);
        const double C2 = 1.118033988749895, D2 = 1.9364916731037085;   // sqrt(1.25), sqrt(3.75)
        const double tau = z == 0 ? 0 : z / (sqrt(R * R + z * z) + R);
        const double ct = 2 * tau / (1 + tau * tau), st = (1 - tau * tau) / (1 + tau * tau);
        const double cc = ct * ct, cs = ct * st, ss = st * st;
        const double Y20 = 3 * C2 * cc - C2, dY20 = -6 * C2 * cs, d2Y20 = -12 * C2 * cc + 6 * C2;
        *val = Y20 * C[i20] + C[i00];
        if(NQ >= 3) { g->dr = Y20 * dC[i20] + dC[i00]; g->dt = dY20 * C[i20]; g->dphi = 0; }
        if(NQ == 6) {
            h->dr2 = Y20 * d2C[i20] + d2C[i00]; h->drdt = dY20 * dC[i20]; h->dt2 = d2Y20 * C[i20];
            h->drdphi = h->dtdphi = h->dphi2 = 0;
        }
        if(ind.mmax == 2) {
            double sp, cp;
            sincos(2 * phi, &sp, &cp);
            const double Y22 = D2 * ss, dY22 = 2 * D2 * cs, d2Y22 = 4 * D2 * cc - 2 * D2;
            *val += Y22 * C[i22] * cp;
            if(NQ >= 3) {
                g->dr += Y22 * dC[i22] * cp; g->dt += dY22 * C[i22] * cp; g->dphi += Y22 * C[i22] * -2 * sp;
            }
            if(NQ == 6) {
                h->dr2 += Y22 * d2C[i22] * cp; h->drdt += dY22 * dC[i22] * cp; h->dt2 += d2Y22 * C[i22] * cp;
                h->drdphi += Y22 * dC[i22] * -2 * sp; h->dtdphi += dY22 * C[i22] * -2 * sp;
                h->dphi2 += Y22 * C[i22] * -4 * cp;
            }
        }
        return;
    }
    double Cm[6 * (2 * LMAX_MAX + 1)];
    double P[LMAX_MAX + 1], dP[LMAX_MAX + 1], d2P[LMAX_MAX + 1];
    const double tau = z == 0 ? 0 : z / (sqrt(R * R + z * z) + R);
    const int nm = ind.mmax - ind.mmin() + 1;
    for(int mm = 0; mm < nm; mm++) {
        const int m = mm + ind.mmin(), lmin = ind.lmin(m);
        if(lmin > ind.lmax) continue;
        const double mul = m == 0 ? 2 * SQRT_PI : 2 * SQRT_PI * M_SQRT2;
        for(int q = 0; q < NQ; q++) Cm[mm + q * nm] = 0;
        const int absm = m < 0 ? -m : m;
        legendreArray(ind.lmax, absm, tau, P, NQ >= 3 ? dP : nullptr, NQ == 6 ? d2P : nullptr);
        for(int l = lmin; l <= ind.lmax; l += ind.step) {
            const int c = HarmIndices::index(l, m), p = l - absm;
            double C, dC = 0, d2C = 0;
            coef(c, &C, &dC, &d2C);
            Cm[mm] += P[p] * C * mul;
            if(NQ >= 3) {
                Cm[mm + nm]     += P[p] * dC * mul;
                Cm[mm + 2 * nm] += dP[p] * C * mul;
            }
            if(NQ == 6) {
                Cm[mm + 3 * nm] += P[p] * d2C * mul;
                Cm[mm + 4 * nm] += dP[p] * dC * mul;
                Cm[mm + 5 * nm] += d2P[p] * C * mul;
            }
        }
    }
    fourierSum<NQ>(ind, phi, Cm, val, g, h);
}

/// chain rule from (ln r, theta, phi) to (R, z, phi); reference transformDerivsSphToCyl :824-848
template<int NQ>
__device__ __forceinline__ void sphToCyl(double R, double z, const SphDerivs& g, const SphHess& h,
    CylDerivs* gc, CylHess* hc)
{
    const double r2inv = 1 / (R * R + z * z);
    const double drdR = R * r2inv, drdz = z * r2inv, dtdR = drdz, dtdz = -drdR;
    gc->dR = g.dr * drdR + g.dt * dtdR;
    gc->dz = g.dr * drdz + g.dt * dtdz;
    gc->dphi = g.dphi;
    if(NQ == 6) {
        const double d2rdR2 = drdz * drdz - drdR * drdR, d2rdRdz = -2 * drdR * drdz, d2rdz2 = -d2rdR2;
        const double d2tdR2 = d2rdRdz, d2tdRdz = -d2rdR2, d2tdz2 = -d2rdRdz;
        hc->dR2 = (h.dr2 * drdR + h.drdt * dtdR) * drdR + (h.drdt * drdR + h.dt2 * dtdR) * dtdR +
                  g.dr * d2rdR2 + g.dt * d2tdR2;
        hc->dRdz = (h.dr2 * drdz + h.drdt * dtdz) * drdR + (h.drdt * drdz + h.dt2 * dtdz) * dtdR +
                   g.dr * d2rdRdz + g.dt * d2tdRdz;
        hc->dz2 = (h.dr2 * drdz + h.drdt * dtdz) * drdz + (h.drdt * drdz + h.dt2 * dtdz) * dtdz +
                  g.dr * d2rdz2 + g.dt * d2tdz2;
        hc->dRdphi = h.drdphi * drdR + h.dtdphi * dtdR;
        hc->dzdphi = h.drdphi * drdz + h.dtdphi * dtdz;
        hc->dphi2 = h.dphi2;
    }
}

/** Power-law asymptotic expansion outside the radial grid; reference PowerLawMultipole::evalCyl,
    src/potential_multipole.cpp:1600-1658. */
template<int NQ>
__device__ void evalPowerLaw(const PowerLawView& A, double R, double z, double phi,
    double* pot, CylDerivs* g, CylHess* h)
{
    const HarmIndices& ind = A.ind;
    const double rsq = R * R + z * z, dlogr = log(rsq / A.r0sq) * 0.5;
    const int lmax = (A.inner && rsq < A.r0sq * 1e-16) || (!A.inner && rsq > A.r0sq * 1e16) ? 0 : ind.lmax;
    // Phi_lm(r) = U (r/r0)^s [ln(r/r0) if s == v] + W (r/r0)^v [+ Q (r/r0)^2]; derivatives in ln r
    auto coef = [&](int c, double* C, double* dC, double* d2C) {
        const int l = static_cast<int>(sqrt(static_cast<double>(c)));
        const double s = ldg(A.S + c), u = ldg(A.U + c), w = ldg(A.W + c), v = A.inner ? l : -l - 1;
        const double rv = v != 0 ? exp(dlogr * v) : 1;
        const double rs = s != v ? (s != 0 ? exp(dlogr * s) : 1) : rv;
        const double urs = u * rs * (s != v || u == 0 ? 1 : dlogr);
        const double wrv = w * rv;
        const double qr2 = v == 0 ? A.Q * rsq / A.r0sq : 0;
        *C = urs + wrv + qr2;
        if(NQ >= 3) *dC = urs * s + wrv * v + (s != v ? 0 : u * rs) + qr2 * 2;
        if(NQ == 6) *d2C = urs * s * s + wrv * v * v + (s != v ? 0 : 2 * s * u * rs) + qr2 * 4;
    };
    if(lmax == 0) {
        double C0, dC0 = 0, d2C0 = 0;
        coef(0, &C0, &dC0, &d2C0);
        *pot = C0;
        const double rsqinv = rsq > 0 ? 1 / rsq : 0;
        const double Rr2 = rsq < INFINITY ? R * rsqinv : 0, zr2 = rsq < INFINITY ? z * rsqinv : 0;
        if(NQ >= 3) { g->dR = dC0 * Rr2; g->dz = dC0 * zr2; g->dphi = 0; }
        if(NQ == 6) {
            const double d2 = d2C0 - 2 * dC0;
            h->dR2 = d2 * Rr2 * Rr2 + dC0 * rsqinv;
            h->dz2 = d2 * zr2 * zr2 + dC0 * rsqinv;
            h->dRdz = d2 * Rr2 * zr2;
            h->dRdphi = h->dzdphi = h->dphi2 = 0;
        }
        return;
    }
    SphDerivs gs; SphHess hs;
    sphHarmInverse<NQ>(ind, R, z, phi, coef, pot, &gs, &hs);
    if(NQ >= 3) sphToCyl<NQ>(R, z, gs, hs, g, h);
}

/** 1-D quintic splines in ln r per (l,m) (lmax <= 2); reference MultipoleInterp1d::evalCyl,
    src/potential_multipole.cpp:1749-1815. */
template<int NQ>
__device__ void evalInterp1d(const MultipoleView& M, double R, double z, double phi,
    double* pot, CylDerivs* g, CylHess* h)
{
    const HarmIndices& ind = M.ind;
    const double r = sqrt(R * R + z * z), logr = log(r);
    double C[9], dC[9], d2C[9];
    const int k = binSearchScaled(logr, M.lnr, M.nr, M.lnrScale);
    auto spline = [&](int c, double* f, double* df, double* d2f) {
        const double* t = M.spl1d + static_cast<size_t>(c) * M.nr * 3;
        if(k < 0 || k >= M.nr - 1) {   // linear extrapolation beyond the grid
            const int e = k < 0 ? 0 : M.nr - 1;
            const double f0 = ldg(t + 3 * e), d0 = ldg(t + 3 * e + 1);
            *f = f0 + (d0 == 0 ? 0 : d0 * (logr - M.lnr[e]));
            if(df) *df = d0;
            if(d2f) *d2f = 0;
            return;
        }
        const double* a = t + 3 * k;
        const double fl[1] = { ldg(a) }, fh[1] = { ldg(a + 3) }, f1l[1] = { ldg(a + 1) }, f1h[1] = { ldg(a + 4) },
            f2l[1] = { ldg(a + 2) }, f2h[1] = { ldg(a + 5) };
        quinticSegmentR<1>(logr, M.lnr[k], M.lnr[k + 1], M.lnrInvH[k], fl, fh, f1l, f1h, f2l, f2h, f, df, d2f);
    };
    spline(0, &C[0], NQ >= 3 ? &dC[0] : nullptr, NQ == 6 ? &d2C[0] : nullptr);
    if(M.logScaling) {
        const double ex = exp(C[0]), P = 1 / (M.invPhi0 - ex);
        C[0] = P;
        if(NQ >= 3) {
            const double dPdX = P * P * ex;
            if(NQ == 6) d2C[0] = dPdX * (d2C[0] + dC[0] * dC[0] * P * (M.invPhi0 + ex));
            dC[0] *= dPdX;
        }
    }
    SphDerivs gs; SphHess hs;
    if(ind.lmax == 0) {
        *pot = C[0];
        gs.dr = NQ >= 3 ? dC[0] : 0; gs.dt = gs.dphi = 0;
        hs.dr2 = NQ == 6 ? d2C[0] : 0; hs.dt2 = hs.dphi2 = hs.drdt = hs.drdphi = hs.dtdphi = 0;
    } else {
        for(int m = ind.mmin(); m <= ind.mmax; m++)
            for(int l = ind.lmin(m); l <= ind.lmax; l += ind.step) {
                const int c = HarmIndices::index(l, m);
                if(c == 0) continue;
                spline(c, &C[c], NQ >= 3 ? &dC[c] : nullptr, NQ == 6 ? &d2C[c] : nullptr);
                if(M.logScaling) {
                    if(NQ == 6) d2C[c] = d2C[c] * C[0] + 2 * dC[c] * dC[0] + C[c] * d2C[0];
                    if(NQ >= 3) dC[c] = dC[c] * C[0] + C[c] * dC[0];
                    C[c] *= C[0];
                }
            }
        auto coef = [&](int c, double* a, double* b, double* d) {
            *a = C[c]; if(NQ >= 3) *b = dC[c]; if(NQ == 6) *d = d2C[c];
        };
        sphHarmInverse<NQ>(ind, R, z, phi, coef, pot, &gs, &hs);
    }
    if(NQ >= 3) sphToCyl<NQ>(R, z, gs, hs, g, h);
}

/** 2-D quintic spline of one harmonic at (x = ln r, y = tau) inside cell (xi, yi): value and
    the requested derivatives.  Reference QuinticSpline2d::evalDeriv, src/math_spline.cpp:2535-2597
    (corner values shifted by one corner value to limit round-off).  xhi, yhi: the tabulated
    reciprocal widths of the cell. */
template<int NQ, bool SPLIT = false>
__device__ __forceinline__ void spline2dCell(const double* tab, int nt, int xi, int yi,
    double x, double xl, double xh, double y, double yl, double yh, double xhi, double yhi,
    double* z, double* zx, double* zy, double* zxx, double* zxy, double* zyy)
{
    const double* nll = tab + (static_cast<size_t>(xi) * nt + yi) * NODE_STRIDE;  // (xlow, ylow)
    const double* nlu = nll + NODE_STRIDE;                                         // (xlow, yupp)
    const double* nul = nll + static_cast<size_t>(nt) * NODE_STRIDE;               // (xupp, ylow)
    const double* nuu = nul + NODE_STRIDE;                                         // (xupp, yupp)
    // node layout: 0 f, 1 fx, 2 fy, 3 fxx, 4 fxy, 5 fyy, 6 fxxy, 7 fxyy, 8 fxxyy (9: padding, not read)
    double F[6], dF[6], d2F[6];
    double off;
    if constexpr(SPLIT) {
        // the y-segments of the lower x nodes (components f, fx, fxx at xl) first, then those of
        // the upper x nodes: half of the cell's values are live at a time (the upper nodes' loads
        // wait for the lower half's first result); every component's arithmetic is unchanged.
        // Fewer registers for callers that hold much state (the root searches); slower for the
        // others, whose loads it serialises
        off = x == xh ? (y == yh ? ldg(nuu) : ldg(nul)) : (y == yh ? ldg(nlu) : ldg(nll));
        auto half = [&](const double* a0, const double* a1, int k0) {
            double p[9], q[9];
#pragma unroll
            for(int m = 0; m < 4; m++) {
                const double2 u = ldg2(a0 + 2 * m), v = ldg2(a1 + 2 * m);
                p[2 * m] = u.x; p[2 * m + 1] = u.y; q[2 * m] = v.x; q[2 * m + 1] = v.y;
            }
            p[8] = ldg(a0 + 8); q[8] = ldg(a1 + 8);
            const double fl[3]  = { p[0] - off, p[1], p[3] }, fu[3]  = { q[0] - off, q[1], q[3] };
            const double f1l[3] = { p[2], p[4], p[6] },       f1u[3] = { q[2], q[4], q[6] };
            const double f2l[3] = { p[5], p[7], p[8] },       f2u[3] = { q[5], q[7], q[8] };
            double G[3], dG[3], d2G[3];
            quinticSegmentR<3>(y, yl, yh, yhi, fl, fu, f1l, f1u, f2l, f2u, G, NQ >= 3 ? dG : nullptr, NQ == 6 ? d2G : nullptr);
#pragma unroll
            for(int c = 0; c < 3; c++) {
                F[2 * c + k0] = G[c];
                if(NQ >= 3) dF[2 * c + k0] = dG[c];
                if(NQ == 6) d2F[2 * c + k0] = d2G[c];
            }
        };
        half(nll, nlu, 0);
        asm volatile("" : "+l"(nul), "+l"(nuu) : "d"(F[0]));
        half(nul, nuu, 1);
    } else {
        double ll[9], lu[9], ul[9], uu[9];
#pragma unroll
        for(int q = 0; q < 4; q++) {
            double2 a = ldg2(nll + 2 * q), b = ldg2(nlu + 2 * q), c = ldg2(nul + 2 * q), d = ldg2(nuu + 2 * q);
            ll[2 * q] = a.x; ll[2 * q + 1] = a.y; lu[2 * q] = b.x; lu[2 * q + 1] = b.y;
            ul[2 * q] = c.x; ul[2 * q + 1] = c.y; uu[2 * q] = d.x; uu[2 * q + 1] = d.y;
        }
        ll[8] = ldg(nll + 8); lu[8] = ldg(nlu + 8); ul[8] = ldg(nul + 8); uu[8] = ldg(nuu + 8);
        off = x == xh ? (y == yh ? uu[0] : ul[0]) : (y == yh ? lu[0] : ll[0]);
        const double fl[6]  = { ll[0] - off, ul[0] - off, ll[1], ul[1], ll[3], ul[3] };
        const double fu[6]  = { lu[0] - off, uu[0] - off, lu[1], uu[1], lu[3], uu[3] };
        const double f1l[6] = { ll[2], ul[2], ll[4], ul[4], ll[6], ul[6] };
        const double f1u[6] = { lu[2], uu[2], lu[4], uu[4], lu[6], uu[6] };
        const double f2l[6] = { ll[5], ul[5], ll[7], ul[7], ll[8], ul[8] };
        const double f2u[6] = { lu[5], uu[5], lu[7], uu[7], lu[8], uu[8] };
        quinticSegmentR<6>(y, yl, yh, yhi, fl, fu, f1l, f1u, f2l, f2u, F, NQ >= 3 ? dF : nullptr, NQ == 6 ? d2F : nullptr);
    }
    quinticSegmentR<1>(x, xl, xh, xhi, &F[0], &F[1], &F[2], &F[3], &F[4], &F[5], z, zx, zxx);
    *z += off;
    if(NQ >= 3)
        quinticSegmentR<1, double>(x, xl, xh, xhi, &dF[0], &dF[1], &dF[2], &dF[3], &dF[4], &dF[5], zy, zxy, nullptr);
    if(NQ == 6)
        quinticSegmentR<1, double>(x, xl, xh, xhi, &d2F[0], &d2F[1], &d2F[2], &d2F[3], &d2F[4], &d2F[5], zyy, nullptr, nullptr);
}

/** The same cell in FP32 (the mixed-precision evaluation of the m != 0 harmonics): node values
    from the FP32 copy of the table, local coordinates x - xl, y - yl formed in FP64 and rounded,
    so that the interpolation keeps FP32 precision relative to the cell size; results in FP64. */
template<int NQ>
__device__ __forceinline__ void spline2dCell32(const float* tab, int nt, int xi, int yi,
    double x, double xl, double xh, double y, double yl, double yh,
    double* z, double* zx, double* zy, double* zxx, double* zxy, double* zyy)
{
    const float* nll = tab + (static_cast<size_t>(xi) * nt + yi) * NODE_STRIDE;
    const float* nlu = nll + NODE_STRIDE;
    const float* nul = nll + static_cast<size_t>(nt) * NODE_STRIDE;
    const float* nuu = nul + NODE_STRIDE;
    float ll[10], lu[10], ul[10], uu[10];
#pragma unroll
    for(int q = 0; q < 5; q++) {
        const float2 a = __ldg(reinterpret_cast<const float2*>(nll) + q), b = __ldg(reinterpret_cast<const float2*>(nlu) + q),
            c = __ldg(reinterpret_cast<const float2*>(nul) + q), d = __ldg(reinterpret_cast<const float2*>(nuu) + q);
        ll[2 * q] = a.x; ll[2 * q + 1] = a.y; lu[2 * q] = b.x; lu[2 * q + 1] = b.y;
        ul[2 * q] = c.x; ul[2 * q + 1] = c.y; uu[2 * q] = d.x; uu[2 * q + 1] = d.y;
    }
    const float hx = static_cast<float>(xh - xl), hy = static_cast<float>(yh - yl);
    const float lx = x == xh ? hx : static_cast<float>(x - xl), ly = y == yh ? hy : static_cast<float>(y - yl);
    const float off = x == xh ? (y == yh ? uu[0] : ul[0]) : (y == yh ? lu[0] : ll[0]);
    const float fl[6]  = { ll[0] - off, ul[0] - off, ll[1], ul[1], ll[3], ul[3] };
    const float fu[6]  = { lu[0] - off, uu[0] - off, lu[1], uu[1], lu[3], uu[3] };
    const float f1l[6] = { ll[2], ul[2], ll[4], ul[4], ll[6], ul[6] };
    const float f1u[6] = { lu[2], uu[2], lu[4], uu[4], lu[6], uu[6] };
    const float f2l[6] = { ll[5], ul[5], ll[7], ul[7], ll[8], ul[8] };
    const float f2u[6] = { lu[5], uu[5], lu[7], uu[7], lu[8], uu[8] };
    float F[6], dF[6], d2F[6], v, vx, vxx, vy, vxy, vyy;
    quinticSegment<6, float>(ly, 0.f, hy, fl, fu, f1l, f1u, f2l, f2u, F, NQ >= 3 ? dF : nullptr, NQ == 6 ? d2F : nullptr);
    quinticSegment<1, float>(lx, 0.f, hx, &F[0], &F[1], &F[2], &F[3], &F[4], &F[5], &v, &vx, &vxx);
    *z = static_cast<double>(v) + static_cast<double>(off);
    *zx = vx; *zxx = vxx;
    if(NQ >= 3) {
        quinticSegment<1, float>(lx, 0.f, hx, &dF[0], &dF[1], &dF[2], &dF[3], &dF[4], &dF[5], &vy, &vxy, nullptr);
        *zy = vy; *zxy = vxy;
    }
    if(NQ == 6) {
        quinticSegment<1, float>(lx, 0.f, hx, &d2F[0], &d2F[1], &d2F[2], &d2F[3], &d2F[4], &d2F[5], &vyy, nullptr, nullptr);
        *zyy = vyy;
    }
}

/** 2-D splines per azimuthal harmonic; reference MultipoleInterp2d::evalCyl,
    src/potential_multipole.cpp:1969-2080. */
template<int NQ>
__device__ void evalInterp2d(const MultipoleView& M, double R, double z, double phi,
    double* pot, CylDerivs* g, CylHess* h)
{
    const HarmIndices& ind = M.ind;
    const double r = sqrt(R * R + z * z), logr = log(r), rpRinv = 1. / (r + fabs(R));
    const double tau = R == 0 ? signOf(z) : z * rpRinv;
    const int mmin = ind.mmin(), nm = ind.mmax - mmin + 1;
    double Cm[6 * (2 * LMAX_MAX + 1)];
    double* Phi = Cm;  double* dlnr = Cm + nm;  double* dtau = Cm + 2 * nm;
    double* dlnr2 = Cm + 3 * nm;  double* dlnrdtau = Cm + 4 * nm;  double* dtau2 = Cm + 5 * nm;
    const int xi = binSearchScaled(logr, M.lnr, M.nr, M.lnrScale), yi = binSearchScaled(tau, M.tau, M.nt, M.tauScale);
    const bool inside = !(xi < 0 || xi >= M.nr - 1 || yi < 0 || yi >= M.nt - 1);
    const double xl = inside ? M.lnr[xi] : 0, xh = inside ? M.lnr[xi + 1] : 0;
    const double yl = inside ? M.tau[yi] : 0, yh = inside ? M.tau[yi + 1] : 0;
    const double xhi = inside ? M.lnrInvH[xi] : 0, yhi = inside ? M.tauInvH[yi] : 0;
    for(int mm = 0; mm < nm; mm++) {
        const int m = mm + mmin;
        if(ind.lmin(m) > ind.lmax) continue;
        if(!inside) {   // out of the table: NaN, as the reference spline does
            for(int q = 0; q < NQ; q++) Cm[mm + q * nm] = NAN;
            continue;
        }
        const double* tab = M.spl2d + static_cast<size_t>(M.splSlot[m + ind.mmax]) * M.nr * M.nt * NODE_STRIDE;
        double dummy;
        spline2dCell<NQ>(tab, M.nt, xi, yi, logr, xl, xh, tau, yl, yh, xhi, yhi, &Phi[mm],
            NQ >= 3 ? &dlnr[mm] : &dummy, NQ >= 3 ? &dtau[mm] : &dummy,
            NQ == 6 ? &dlnr2[mm] : &dummy, NQ == 6 ? &dlnrdtau[mm] : &dummy, NQ == 6 ? &dtau2[mm] : &dummy);
    }
    if(M.logScaling) {
        const int z0 = -mmin;
        const double ex = exp(Phi[z0]), val = 1 / (M.invPhi0 - ex);
        Phi[z0] = val;
        if(NQ >= 3) {
            const double dPdX = val * val * ex;
            if(NQ == 6) {
                const double d2PdX2 = dPdX * val * (M.invPhi0 + ex);
                dlnr2[z0]    = dPdX * dlnr2[z0]    + d2PdX2 * dlnr[z0] * dlnr[z0];
                dtau2[z0]    = dPdX * dtau2[z0]    + d2PdX2 * dtau[z0] * dtau[z0];
                dlnrdtau[z0] = dPdX * dlnrdtau[z0] + d2PdX2 * dlnr[z0] * dtau[z0];
            }
            dlnr[z0] *= dPdX;
            dtau[z0] *= dPdX;
        }
        for(int mm = 0; mm < nm; mm++) {
            const int m = mm + mmin;
            if(m == 0 || ind.lmin(m) > ind.lmax) continue;
            if(NQ == 6) {
                dlnr2[mm] = dlnr2[mm] * Phi[z0] + Phi[mm] * dlnr2[z0] + 2 * dlnr[mm] * dlnr[z0];
                dtau2[mm] = dtau2[mm] * Phi[z0] + Phi[mm] * dtau2[z0] + 2 * dtau[mm] * dtau[z0];
                dlnrdtau[mm] = dlnrdtau[mm] * Phi[z0] + Phi[mm] * dlnrdtau[z0] +
                               dlnr[mm] * dtau[z0] + dtau[mm] * dlnr[z0];
            }
            if(NQ >= 3) {
                dlnr[mm] = dlnr[mm] * Phi[z0] + Phi[mm] * dlnr[z0];
                dtau[mm] = dtau[mm] * Phi[z0] + Phi[mm] * dtau[z0];
            }
            Phi[mm] *= Phi[z0];
        }
    }
    SphDerivs gs; SphHess hs;
    fourierSum<NQ>(ind, phi, Cm, pot, &gs, &hs);
    if(NQ == 1) return;
    const double rinv = 1 / r, r2inv = rinv * rinv;
    const double drdR = R * r2inv, drdz = z * r2inv, dtdR = -tau * rinv, dtdz = rinv - rpRinv;
    g->dR = gs.dr * drdR + gs.dt * dtdR;
    g->dz = gs.dr * drdz + gs.dt * dtdz;
    g->dphi = gs.dphi;
    if(NQ == 6) {
        const double d2rdR2 = drdz * drdz - drdR * drdR, d2rdRdz = -2 * drdR * drdz, d2rdz2 = -d2rdR2;
        const double d2tdR2 = z * r2inv * rinv;
        const double d2tdRdz = dtdR * dtdR - drdR * drdR * r * rpRinv;
        const double d2tdz2 = -d2tdR2 - dtdR * rpRinv;
        h->dR2 = (hs.dr2 * drdR + hs.drdt * dtdR) * drdR + (hs.drdt * drdR + hs.dt2 * dtdR) * dtdR +
                 gs.dr * d2rdR2 + gs.dt * d2tdR2;
        h->dRdz = (hs.dr2 * drdz + hs.drdt * dtdz) * drdR + (hs.drdt * drdz + hs.dt2 * dtdz) * dtdR +
                  gs.dr * d2rdRdz + gs.dt * d2tdRdz;
        h->dz2 = (hs.dr2 * drdz + hs.drdt * dtdz) * drdz + (hs.drdt * drdz + hs.dt2 * dtdz) * dtdz +
                 gs.dr * d2rdz2 + gs.dt * d2tdz2;
        h->dRdphi = hs.drdphi * drdR + hs.dtdphi * dtdR;
        h->dzdphi = hs.drdphi * drdz + hs.dtdphi * dtdz;
        h->dphi2 = hs.dphi2;
    }
}

/// the lanes of this lane's group of G consecutive lanes
template<int G>
__device__ __forceinline__ unsigned groupMask()
{
    if(G >= 32) return 0xffffffffu;
    const unsigned lane = threadIdx.x & 31;
    return ((1u << G) - 1) << (lane & ~(G - 1));
}

/** The same 2-D spline evaluation with the harmonics held in registers: at most MAXS non-empty
    azimuthal harmonics, listed in M.fastM / M.fastSlot with m = 0 first and the others in
    ascending m (the order in which the reference sums them), so every array index is a
    compile-time constant after unrolling and nothing goes to local memory.  cos/sin(|m| phi)
    come from the same multiple-angle recurrence as trigMultiAngle.
    MIXED: the m != 0 harmonics from the FP32 table in FP32 arithmetic (their sum in FP64).
    G > 1: the evaluation is shared by a group of G consecutive lanes that evaluate the same
    point: lane j of the group evaluates the harmonics s = j, j + G, ..., the m = 0 terms are
    broadcast from lane 0, every scaled harmonic is then broadcast from the lane that evaluated
    it, and every lane forms the Fourier sums itself in the order m = 0, then ascending m.  The
    arithmetic of each harmonic and of the sums is that of G = 1, so every G gives the same bits. */
template<int NQ, int MAXS, int G = 1, bool MIXED = false, bool SPLIT = false>
__device__ __forceinline__ void evalInterp2dFast(const MultipoleView& M, double R, double z, double phi,
    double* pot, CylDerivs* g, CylHess* h)
{
    const int gl = G > 1 ? static_cast<int>(threadIdx.x % G) : 0;
    const unsigned gmask = G > 1 ? groupMask<G>() : 0u;
    const double r = sqrt(R * R + z * z), logr = log(r), rpRinv = 1. / (r + fabs(R));
    const double tau = R == 0 ? signOf(z) : z * rpRinv;
    const int xi = binSearchScaled(logr, M.lnr, M.nr, M.lnrScale), yi = binSearchScaled(tau, M.tau, M.nt, M.tauScale);
    const bool inside = !(xi < 0 || xi >= M.nr - 1 || yi < 0 || yi >= M.nt - 1);
    const int xs = inside ? xi : 0, ys = inside ? yi : 0;
    const double xl = M.lnr[xs], xh = M.lnr[xs + 1], yl = M.tau[ys], yh = M.tau[ys + 1];
    const double xhi = M.lnrInvH[xs], yhi = M.tauInvH[ys];
    const size_t slotStride = static_cast<size_t>(M.nr) * M.nt * NODE_STRIDE;
    double P[MAXS], Dr[MAXS], Dt[MAXS], Drr[MAXS], Drt[MAXS], Dtt[MAXS];
#pragma unroll
    for(int s = 0; s < MAXS; s++) {
        P[s] = Dr[s] = Dt[s] = Drr[s] = Drt[s] = Dtt[s] = 0;
        if(s < M.nFast && s % G == gl) {
            if(MIXED && s > 0)      // m != 0 (angular) harmonics in FP32, the radial m = 0 one in FP64
                spline2dCell32<NQ>(M.spl2d32 + M.fastSlot[s] * slotStride, M.nt, xs, ys, logr, xl, xh, tau, yl, yh,
                    &P[s], &Dr[s], &Dt[s], &Drr[s], &Drt[s], &Dtt[s]);
            else
                spline2dCell<NQ, SPLIT>(M.spl2d + M.fastSlot[s] * slotStride, M.nt, xs, ys, logr, xl, xh, tau, yl, yh,
                    xhi, yhi, &P[s], &Dr[s], &Dt[s], &Drr[s], &Drt[s], &Dtt[s]);
            if(!inside) P[s] = Dr[s] = Dt[s] = Drr[s] = Drt[s] = Dtt[s] = NAN;
        }
    }
    if(G > 1) {     // every lane needs the m = 0 harmonic (log scaling, Fourier sum)
        P[0] = __shfl_sync(gmask, P[0], 0, G);
        if(NQ >= 3) { Dr[0] = __shfl_sync(gmask, Dr[0], 0, G); Dt[0] = __shfl_sync(gmask, Dt[0], 0, G); }
        if(NQ == 6) {
            Drr[0] = __shfl_sync(gmask, Drr[0], 0, G); Drt[0] = __shfl_sync(gmask, Drt[0], 0, G);
            Dtt[0] = __shfl_sync(gmask, Dtt[0], 0, G);
        }
    }
    if(M.logScaling) {
        const double ex = exp(P[0]), val = 1 / (M.invPhi0 - ex);
        P[0] = val;
        if(NQ >= 3) {
            const double dPdX = val * val * ex;
            if(NQ == 6) {
                const double d2PdX2 = dPdX * val * (M.invPhi0 + ex);
                Drr[0] = dPdX * Drr[0] + d2PdX2 * Dr[0] * Dr[0];
                Dtt[0] = dPdX * Dtt[0] + d2PdX2 * Dt[0] * Dt[0];
                Drt[0] = dPdX * Drt[0] + d2PdX2 * Dr[0] * Dt[0];
            }
            Dr[0] *= dPdX;
            Dt[0] *= dPdX;
        }
#pragma unroll
        for(int s = 1; s < MAXS; s++) {
            if(s < M.nFast && s % G == gl) {
                if(NQ == 6) {
                    Drr[s] = Drr[s] * P[0] + P[s] * Drr[0] + 2 * Dr[s] * Dr[0];
                    Dtt[s] = Dtt[s] * P[0] + P[s] * Dtt[0] + 2 * Dt[s] * Dt[0];
                    Drt[s] = Drt[s] * P[0] + P[s] * Drt[0] + Dr[s] * Dt[0] + Dt[s] * Dr[0];
                }
                if(NQ >= 3) {
                    Dr[s] = Dr[s] * P[0] + P[s] * Dr[0];
                    Dt[s] = Dt[s] * P[0] + P[s] * Dt[0];
                }
                P[s] *= P[0];
            }
        }
    }
    if(G > 1) {     // every lane gets every harmonic from the lane that evaluated it
#pragma unroll
        for(int s = 1; s < MAXS; s++) {
            if(s < M.nFast) {
                P[s] = __shfl_sync(gmask, P[s], s % G, G);
                if(NQ >= 3) { Dr[s] = __shfl_sync(gmask, Dr[s], s % G, G); Dt[s] = __shfl_sync(gmask, Dt[s], s % G, G); }
                if(NQ == 6) {
                    Drr[s] = __shfl_sync(gmask, Drr[s], s % G, G); Drt[s] = __shfl_sync(gmask, Drt[s], s % G, G);
                    Dtt[s] = __shfl_sync(gmask, Dtt[s], s % G, G);
                }
            }
        }
    }
    // Fourier synthesis in the reference's order: m = 0, then the others by ascending m
    SphDerivs gs; SphHess hs;
    *pot = P[0];
    if(NQ >= 3) { gs.dr = Dr[0]; gs.dt = Dt[0]; gs.dphi = 0; }
    if(NQ == 6) {
        hs.dr2 = Drr[0]; hs.drdt = Drt[0]; hs.dt2 = Dtt[0];
        hs.drdphi = hs.dtdphi = hs.dphi2 = 0;
    }
    if(MAXS > 1 && M.nFast > 1) {
        double cm[MAXS], sm[MAXS];
        double s1, c1, sh, ch;
        sincos(phi, &s1, &c1);
        sincos(0.5 * phi, &sh, &ch);
        const double alpha = 2 * sh * sh, beta = s1;
        double cp = 1, sp = 0;
#pragma unroll
        for(int k = 1; k <= LMAX_MAX; k++) {
            if(k <= M.ind.mmax) {
                const double c = cp - (alpha * cp + beta * sp), sv = sp - (alpha * sp - beta * cp);
#pragma unroll
                for(int s = 1; s < MAXS; s++)
                    if(M.fastM[s] == k || M.fastM[s] == -k) { cm[s] = c; sm[s] = sv; }
                cp = c;
                sp = sv;
            }
        }
#pragma unroll
        for(int s = 1; s < MAXS; s++) {
            if(s < M.nFast) {
                const int m = M.fastM[s];
                const double tr = m > 0 ? cm[s] : sm[s];
                const double dtr = m > 0 ? -m * sm[s] : -m * cm[s];
                const double d2tr = -m * m * tr;
                *pot += P[s] * tr;
                if(NQ >= 3) {
                    gs.dr += Dr[s] * tr;
                    gs.dt += Dt[s] * tr;
                    gs.dphi += P[s] * dtr;
                }
                if(NQ == 6) {
                    hs.dr2 += Drr[s] * tr;
                    hs.drdt += Drt[s] * tr;
                    hs.dt2 += Dtt[s] * tr;
                    hs.drdphi += Dr[s] * dtr;
                    hs.dtdphi += Dt[s] * dtr;
                    hs.dphi2 += P[s] * d2tr;
                }
            }
        }
    }
    if(NQ == 1) return;
    const double rinv = 1 / r, r2inv = rinv * rinv;
    const double drdR = R * r2inv, drdz = z * r2inv, dtdR = -tau * rinv, dtdz = rinv - rpRinv;
    g->dR = gs.dr * drdR + gs.dt * dtdR;
    g->dz = gs.dr * drdz + gs.dt * dtdz;
    g->dphi = gs.dphi;
    if(NQ == 6) {
        const double d2rdR2 = drdz * drdz - drdR * drdR, d2rdRdz = -2 * drdR * drdz, d2rdz2 = -d2rdR2;
        const double d2tdR2 = z * r2inv * rinv;
        const double d2tdRdz = dtdR * dtdR - drdR * drdR * r * rpRinv;
        const double d2tdz2 = -d2tdR2 - dtdR * rpRinv;
        h->dR2 = (hs.dr2 * drdR + hs.drdt * dtdR) * drdR + (hs.drdt * drdR + hs.dt2 * dtdR) * dtdR +
                 gs.dr * d2rdR2 + gs.dt * d2tdR2;
        h->dRdz = (hs.dr2 * drdz + hs.drdt * dtdz) * drdR + (hs.drdt * drdz + hs.dt2 * dtdz) * dtdR +
                  gs.dr * d2rdRdz + gs.dt * d2tdRdz;
        h->dz2 = (hs.dr2 * drdz + hs.drdt * dtdz) * drdz + (hs.drdt * drdz + hs.dt2 * dtdz) * dtdz +
                 gs.dr * d2rdz2 + gs.dt * d2tdz2;
        h->dRdphi = hs.drdphi * drdR + hs.dtdphi * dtdR;
        h->dzdphi = hs.drdphi * drdz + hs.dtdphi * dtdz;
        h->dphi2 = hs.dphi2;
    }
}

/// which spline evaluators a kernel instantiation includes
enum EvalKind {
    EVAL_GENERAL = 0,   ///< any Multipole (runtime dispatch, local-memory harmonic arrays)
    EVAL_AXI = 1,       ///< axisymmetric: a single (m = 0) harmonic in registers
    EVAL_FAST = 2       ///< up to FAST_MAX_HARMONICS harmonics in registers
};

/** Multipole::evalCyl: pick the inner asymptote, the spline interpolator or the outer
    asymptote by radius (reference src/potential_multipole.cpp:1538-1548).
    NQ = 1 (value), 3 (+ gradient) or 6 (+ Hessian); KIND selects the spline evaluator
    (the host picks the instantiation that matches the potential). */
template<int NQ, int KIND = EVAL_GENERAL, int G = 1, bool MIXED = false, bool SPLIT = false>
__device__ __forceinline__ void evalMultipoleCyl(const MultipoleView& M, double R, double z, double phi,
    double* pot, CylDerivs* g, CylHess* h)
{
    static_assert(G == 1 || KIND == EVAL_FAST, "the group-shared evaluation is that of the multi-harmonic kind");
    const double rsq = R * R + z * z;
    if(rsq < M.rInnerSq)
        evalPowerLaw<NQ>(M.inner, R, z, phi, pot, g, h);
    else if(rsq > M.rOuterSq)
        evalPowerLaw<NQ>(M.outer, R, z, phi, pot, g, h);
    else if(M.is2d) {
        if(KIND == EVAL_AXI)
            evalInterp2dFast<NQ, 1, 1, false, SPLIT>(M, R, z, phi, pot, g, h);
        else if(KIND == EVAL_FAST)
            evalInterp2dFast<NQ, FAST_MAX_HARMONICS, G, MIXED>(M, R, z, phi, pot, g, h);
        else
            evalInterp2d<NQ>(M, R, z, phi, pot, g, h);
    } else
        evalInterp1d<NQ>(M, R, z, phi, pot, g, h);
}

/// out-of-line copy of evalMultipoleCyl: callers with many call sites (root finders, stage
/// loops) share one body instead of inlining it at every site
template<int NQ, int KIND>
__device__ __noinline__ void evalMultipoleCylCall(const MultipoleView& M, double R, double z, double phi,
    double* pot, CylDerivs* g, CylHess* h)
{
    evalMultipoleCyl<NQ, KIND>(M, R, z, phi, pot, g, h);
}

/// the evaluator kind matching a potential (host side)
inline int evalKindOf(const MultipoleView& M)
{
    if(!M.is2d || M.nFast == 0) return EVAL_GENERAL;
    return M.nFast == 1 ? EVAL_AXI : EVAL_FAST;
}

/** Evaluation at a Cartesian point with gradient (and Hessian xx,yy,zz,xy,yz,zx) in Cartesian
    coordinates: Car -> Cyl -> evaluate -> back (reference coord::evalAndConvert,
    src/coord.h:831-856, with the Car<->Cyl derivatives of src/coord.cpp:94-123, 608-719). */
template<int NQ, int KIND = EVAL_GENERAL, int G = 1, bool MIXED = false>
__device__ __forceinline__ void evalMultipoleCar(const MultipoleView& M, double x, double y, double z,
    double* pot, double* grad, double* hess)
{
    const double R2 = x * x + y * y, R = sqrt(R2);
    // a potential with only m = 0 terms (its splines and both asymptotes): its evaluators neither
    // read the azimuth nor give a phi derivative (exactly 0), so neither atan2 nor the azimuth's
    // derivatives are formed (the results are the same bits)
    const bool noAzimuth = KIND == EVAL_AXI && NQ <= 3 && M.ind.mmax == 0 && M.inner.ind.mmax == 0 &&
                           M.outer.ind.mmax == 0;
    double phi, cphi, sphi;
    double dRdx, dRdy, dphidx = 0, dphidy = 0;
    if(R == 0) {
        phi = 0; dRdx = dRdy = dphidx = dphidy = 1;
        cphi = sphi = 1;
    } else {
        cphi = x / R; sphi = y / R;
        dRdx = cphi; dRdy = sphi;
        if(!noAzimuth) { dphidx = -sphi / R; dphidy = cphi / R; }
        phi = noAzimuth ? 0 : atan2(y, x);
    }
    CylDerivs g; CylHess h;
    evalMultipoleCyl<NQ, KIND, G, MIXED>(M, R, z, phi, pot, &g, &h);
    if(NQ >= 3) {
        grad[0] = noAzimuth ? g.dR * dRdx : g.dR * dRdx + g.dphi * dphidx;
        grad[1] = noAzimuth ? g.dR * dRdy : g.dR * dRdy + g.dphi * dphidy;
        grad[2] = g.dz;
    }
    if(NQ == 6) {
        double d2Rdx2, d2Rdy2, d2Rdxdy, d2phidx2, d2phidy2, d2phidxdy;
        if(R == 0) {
            d2Rdx2 = d2Rdy2 = d2Rdxdy = d2phidx2 = d2phidy2 = d2phidxdy = 1;
        } else {
            d2Rdx2 = sphi * sphi / R; d2Rdy2 = cphi * cphi / R; d2Rdxdy = -sphi * cphi / R;
            d2phidx2 = 2 * sphi * cphi / R2; d2phidy2 = -d2phidx2; d2phidxdy = (sphi * sphi - cphi * cphi) / R2;
        }
        hess[0] = (h.dR2 * dRdx + h.dRdphi * dphidx) * dRdx + (h.dRdphi * dRdx + h.dphi2 * dphidx) * dphidx +
                  g.dR * d2Rdx2 + g.dphi * d2phidx2;                                         // xx
        hess[1] = (h.dR2 * dRdy + h.dRdphi * dphidy) * dRdy + (h.dRdphi * dRdy + h.dphi2 * dphidy) * dphidy +
                  g.dR * d2Rdy2 + g.dphi * d2phidy2;                                         // yy
        hess[2] = h.dz2;                                                                      // zz
        hess[3] = (h.dR2 * dRdy + h.dRdphi * dphidy) * dRdx + (h.dRdphi * dRdy + h.dphi2 * dphidy) * dphidx +
                  g.dR * d2Rdxdy + g.dphi * d2phidxdy;                                       // xy
        hess[4] = h.dRdz * dRdy + h.dzdphi * dphidy;                                          // yz
        hess[5] = h.dRdz * dRdx + h.dzdphi * dphidx;                                          // zx
    }
}

}  // namespace agb
