// Focal distance from shell orbits, on the device (one (E, Lz) node per thread).
//
// Reference: actions::estimateFocalDistanceShellOrbit and findCrossingPointR
// (src/actions_focal_distance_finder.cpp:86-297), the radius routines of potential_utils
// (R_circ, R_max, v_circ, innerSlope, findPlanarOrbitExtent, refineRoot;
// src/potential_utils.cpp:228-729) and the DOP853 stepper with dense output
// (src/math_ode.cpp:35-426), here for the 8-D meridional-plane system with its variational
// equations.  All potential evaluations are in the equatorial plane or the meridional plane of an
// axisymmetric Multipole.
#pragma once
#include "dop853.cuh"

namespace agb {

constexpr double SHELL_ACCURACY_ROOT = 1e-10;       // potential_utils.cpp:31
constexpr double SHELL_HUGE_NUMBER = 1e100;          // potential_utils.cpp:40
constexpr double SHELL_MIN_REL_DIFFERENCE = 3.666852862501036e-11;   // DBL_EPSILON / DBL_EPSILON^(1/3)
constexpr double SHELL_LREL_NEARLY_CIRCULAR = 0.999999;             // potential_utils.cpp:50
constexpr double SHELL_ACCURACY_RSHELL = 1e-6;       // actions_focal_distance_finder.cpp:17
constexpr double SHELL_ACCURACY_INTEGR = 1e-8;       // actions_focal_distance_finder.cpp:19
constexpr int SHELL_MAX_NUM_STEPS_ODE = 200;         // actions_focal_distance_finder.cpp:21

/// potential and its first two R-derivatives in the equatorial plane (Axisymmetrized::evalDeriv)
__device__ __forceinline__ void axiEvalR(const MultipoleView& M, double R, double* val, double* der, double* der2)
{
    double Phi;
    CylDerivs g; CylHess h;
    if(der2)     evalMultipoleCylCall<6, EVAL_AXI>(M, R, 0, 0, &Phi, &g, &h);
    else if(der) evalMultipoleCylCall<3, EVAL_AXI>(M, R, 0, 0, &Phi, &g, &h);
    else         evalMultipoleCylCall<1, EVAL_AXI>(M, R, 0, 0, &Phi, &g, &h);
    if(val) *val = Phi;
    if(der) *der = g.dR;
    if(der2) *der2 = h.dR2;
}

/// root finding in u in (-inf, inf) through s in [0, 1] (ScaledFnc<ScalingInf>, math_core.h:214-232)
template<class F>
struct ScaledInf {
    static constexpr bool hasDeriv = F::hasDeriv;
    const F& f;
    __device__ void operator()(double s, double* v, double* d) const {
        double duds;
        const double u = unscaleInf(s, d ? &duds : nullptr);
        double dfdu = NAN;
        f(u, v, d ? &dfdu : nullptr);
        if(d) *d = dfdu * duds;
    }
};
template<class F>
__device__ double findRootInf(const F& f, double tol)
{
    ScaledInf<F> sf{ f };
    return unscaleInf(findRoot(sf, 0, 1, tol), nullptr);
}

/// the potential of an axisymmetric Multipole and its R-derivatives in the equatorial plane, as
/// the evaluator object of the radius routines below (any type with this call operator works)
struct AxiRadial {
    const MultipoleView* M;
    __device__ void operator()(double R, double* val, double* der, double* der2) const { axiEvalR(*M, R, val, der, der2); }
};

/// Phi(R) + R/2 dPhi/dR = E in ln R (RcircRootFinder, potential_utils.cpp:262-288)
template<class EV>
struct RcircFn {
    static constexpr bool hasDeriv = true;
    EV ev; double E;
    __device__ void operator()(double logR, double* val, double* der) const {
        const double R = exp(logR);
        double Phi, dR, d2R;
        ev(R, &Phi, &dR, der ? &d2R : nullptr);
        if(val) {
            const double v = 0.5 * R * dR;
            *val = Phi - E + (isFinite(v) ? v : 0);
            if(!isFinite(*val)) {
                if(E == -INFINITY) *val = Phi == E ? 0 : 1.0;
                else if(Phi == -INFINITY) *val = -1.0;
                else if(R >= SHELL_HUGE_NUMBER) *val = 1.0;
            }
        }
        if(der) *der = (1.5 * dR + 0.5 * R * d2R) * R;
    }
};

/// Phi(R) = E in ln R (RmaxRootFinder, potential_utils.cpp:232-256)
template<class EV>
struct RmaxFn {
    static constexpr bool hasDeriv = true;
    EV ev; double E;
    __device__ void operator()(double logR, double* val, double* der) const {
        const double R = exp(logR);
        double Phi, dR;
        ev(R, &Phi, der ? &dR : nullptr, nullptr);
        if(val) {
            *val = Phi - E;
            if(!isFinite(*val)) {
                if(E == -INFINITY) *val = Phi == E ? 0 : 1.0;
                else if(Phi == -INFINITY) *val = -1.0;
                else if(R >= SHELL_HUGE_NUMBER) *val = 1.0;
            }
        }
        if(der) *der = dR * R;
    }
};

/// L^2 - R^3 dPhi/dR in ln R (RfromLRootFinder, potential_utils.cpp:290-313)
template<class EV>
struct RfromLFn {
    static constexpr bool hasDeriv = true;
    EV ev; double L2;
    __device__ void operator()(double logR, double* val, double* der) const {
        const double R = exp(logR);
        double dR, d2R;
        ev(R, nullptr, &dR, der ? &d2R : nullptr);
        const double F = R * R * R * dR;
        if(val) *val = isFinite(F) ? F - L2 : (R < 1 ? -L2 : L2);
        if(der) *der = R * R * R * (3 * dR + R * d2R);
    }
};

/// R_circ(E), R_max(E), R_from_Lz(L) (potential_utils.cpp:617-633)
template<class EV>
__device__ double radiusCirc(const EV& ev, double E) { RcircFn<EV> f{ ev, E }; return exp(findRootInf(f, SHELL_ACCURACY_ROOT)); }
template<class EV>
__device__ double radiusMax(const EV& ev, double E) { RmaxFn<EV> f{ ev, E }; return exp(findRootInf(f, SHELL_ACCURACY_ROOT)); }
template<class EV>
__device__ double radiusFromLz(const EV& ev, double L)
{
    if(L == 0) return 0;
    if(fabs(L) == INFINITY) return INFINITY;
    RfromLFn<EV> f{ ev, L * L };
    return exp(findRootInf(f, SHELL_ACCURACY_ROOT));
}

static __device__ double shellRcirc(const MultipoleView& M, double E) { return radiusCirc(AxiRadial{ &M }, E); }
static __device__ double shellRmax(const MultipoleView& M, double E) { return radiusMax(AxiRadial{ &M }, E); }
static __device__ double shellVcirc(const MultipoleView& M, double R)
{
    double Phi, dR;
    if(R == 0) { axiEvalR(M, 0, &Phi, nullptr, nullptr); return isFinite(Phi) ? 0 : INFINITY; }
    axiEvalR(M, R, nullptr, &dR, nullptr);
    return sqrt(R * dR);
}

/// (E - Phi) R^2 - L^2/2 (RPeriApoRootFinder, potential_utils.cpp:315-330)
template<class EV>
struct PeriApoFn {
    static constexpr bool hasDeriv = true;
    EV ev; double E, halfL2;
    __device__ void operator()(double R, double* val, double* der) const {
        double Phi = 0, dR = 0;
        ev(R, &Phi, der ? &dR : nullptr, nullptr);
        if(val) *val = (R > 0 ? (E - Phi) * R * R : 0) - halfL2;
        if(der) *der = 2 * R * (E - Phi) - R * R * dR;
    }
};

/// the same for a power-law potential near the centre (RPeriApoRootFinderPowerLaw, :334-350)
struct PeriApoPowerLawFn {
    static constexpr bool hasDeriv = true;
    double s, v2;
    __device__ void operator()(double x, double* val, double* der) const {
        if(val) *val = s != 0 ? (2 + s) * x * x - 2 * pow(x, 2 + s) - v2 * s : (x == 0 ? 0 : x * x * (1 - 2 * log(x)) - v2);
        if(der) *der = s != 0 ? (4 + 2 * s) * (x - pow(x, 1 + s)) : -4 * x * log(x);
    }
};

/// Halley refinement of a peri/apocentre radius (refineRoot, potential_utils.cpp:355-365)
template<class EV>
__device__ double refinePeriApo(const EV& ev, double R, double E, double L)
{
    double val, der, der2;
    ev(R, &val, &der, &der2);
    const double F = E - val - 0.5 * pow2(L / R);
    const double Fp = pow2(L / R) / R - der;
    const double Fpp = -3 * pow2(L / (R * R)) - der2;
    const double dR = -F / (Fp - 0.5 * F * Fpp / Fp);
    return fabs(dR) < 0.25 * R ? R + dR : R;
}

/// pericentre and apocentre radii of a planar orbit (findPlanarOrbitExtent, potential_utils.cpp:663-729)
template<class EV>
__device__ void planarOrbitExtent(const EV& ev, double E, double L, double& R1, double& R2)
{
    // innerSlope (potential_utils.cpp:647-661) at r = 1e-10
    const double r = 1e-10;
    double Phi, dPhidR, d2PhidR2;
    ev(r, &Phi, &dPhidR, &d2PhidR2);
    const double slope = 1 + r * d2PhidR2 / dPhidR;
    const double coef = slope == 0 ? dPhidR * r : dPhidR / slope * pow(r, 1 - slope);
    const double Phi0 = slope == 0 ? Phi - r * dPhidR * log(r) : Phi - r * dPhidR / slope;
    if(slope > 0 && E >= Phi0 && E < Phi0 * (1 - SHELL_MIN_REL_DIFFERENCE)) {
        const double Rc = slope == 0 ? exp((E - Phi0) / coef - 0.5) : pow((E - Phi0) / (coef * (1 + 0.5 * slope)), 1 / slope);
        if(!isFinite(Rc)) { R1 = R2 = NAN; return; }
        if(Rc == 0) { R1 = R2 = 0; return; }
        const double Lc = Rc * (slope == 0 ? sqrt(coef) : sqrt(coef * slope) * pow(Rc, 0.5 * slope));
        if(L < Lc) {
            PeriApoPowerLawFn f{ slope, pow2(L / Lc) };
            R1 = Rc * fmin(1., findRoot(f, 0, 1, SHELL_ACCURACY_ROOT));
            R2 = Rc * fmax(1., findRoot(f, 1, 2, SHELL_ACCURACY_ROOT));
        } else
            R1 = R2 = Rc;
        return;
    }
    const double Rc = radiusCirc(ev, E);
    if(!isFinite(Rc)) { R1 = R2 = NAN; return; }
    if(Rc == 0) { R1 = R2 = 0; return; }
    double P, dR, d2R;
    ev(Rc, &P, &dR, &d2R);
    const double Lc = Rc * sqrt(Rc * dR);
    if(L >= Lc || (!isFinite(Lc) && Rc <= 1. / SHELL_HUGE_NUMBER)) {
        R1 = R2 = Rc;
    } else if(L > Lc * SHELL_LREL_NEARLY_CIRCULAR || (E - P) * pow2(Rc) <= 0.5 * L * L) {
        const double off = sqrt((1 - pow2(L / Lc)) * dR / (3 * dR + Rc * d2R));
        R1 = Rc * (1 - off);
        R2 = Rc * (1 + off);
        R1 = fmin(Rc, refinePeriApo(ev, R1, E, L));
        R2 = fmax(Rc, refinePeriApo(ev, R2, E, L));
    } else {
        PeriApoFn<EV> f{ ev, E, 0.5 * L * L };
        R1 = findRoot(f, 0, Rc, SHELL_ACCURACY_ROOT);
        R2 = findRoot(f, Rc, 3 * Rc, SHELL_ACCURACY_ROOT);
        if(!isFinite(R2))
            R2 = findRoot(f, Rc, (1 + SHELL_ACCURACY_ROOT) * radiusMax(ev, E), SHELL_ACCURACY_ROOT);
    }
}

static __device__ void shellPlanarExtent(const MultipoleView& M, double E, double L, double& R1, double& R2)
{
    planarOrbitExtent(AxiRadial{ &M }, E, L, R1, R2);
}

/// meridional-plane orbit with its deviation vector: (R, z, vR, vz, dR, dz, dvR, dvz)
/// (OrbitIntegratorMeridionalPlane::eval, actions_focal_distance_finder.cpp:86-113)
struct MeridionalRHS {
    const MultipoleView* M;
    double Lz2;
    __device__ void operator()(const double* x, double* dxdt) const {
        const double signR = x[0] >= 0 ? 1 : -1, R = fabs(x[0]);
        double Phi;
        CylDerivs g; CylHess h;
        evalMultipoleCylCall<6, EVAL_AXI>(*M, R, x[1], 0, &Phi, &g, &h);
        const double Lz2ovR4 = Lz2 > 0 ? Lz2 / pow2(pow2(R)) : 0;
        dxdt[0] = x[2];
        dxdt[1] = x[3];
        dxdt[2] = -(g.dR - Lz2ovR4 * R) * signR;
        dxdt[3] = -g.dz;
        dxdt[4] = x[6];
        dxdt[5] = x[7];
        dxdt[6] = -(h.dR2 + 3 * Lz2ovR4) * x[4] - h.dRdz * signR * x[5];
        dxdt[7] = -h.dRdz * signR * x[4] - h.dz2 * x[5];
    }
};

/// DOP853 on an N-dimensional autonomous system with dense output (OdeStepperDOP853, accAbs = 0,
/// accuracy factor 1): state x, derivative k1, interpolation coefficients r[8]
template<int N, class RHS>
struct Dop853Dense {
    const RHS& f;
    double accRel;
    double x[N], k1[N], r[8][N];
    double prevStep = 0, nextStep = 0;

    __device__ void init(const double* x0)
    {
        for(int i = 0; i < N; i++) x[i] = x0[i];
        f(x, k1);
        // initTimeStep (src/math_ode.cpp:35-91)
        double nx = 0, nd = 0;
        for(int i = 0; i < N; i++) { nx += x[i] * x[i]; nd += k1[i] * k1[i]; }
        const double h1 = fmax(1e-12, fmin(1e12, sqrt(nx / nd) * 0.01));
        double xt[N], k2[N], k3[N];
        for(int i = 0; i < N; i++) xt[i] = x[i] + h1 * k1[i];
        f(xt, k2);
        for(int i = 0; i < N; i++) xt[i] = x[i] + 0.5 * h1 * (k1[i] + k2[i]);
        f(xt, k3);
        double h2 = INFINITY;
        for(int i = 0; i < N; i++) {
            const double d0 = fmax(0., fmax(fabs(x[i]), fabs(xt[i])));
            const double d1 = fmax(fabs(k1[i]), fabs(k3[i]));
            const double d2 = fabs((3 * k2[i] - k1[i] - 2 * k3[i]) / h1);
            const double d3 = fabs(6 * (k3[i] - k2[i]) / (h1 * h1));
            h2 = fmin(h2, (d0 * d2 + d1 * d1) / (d1 * d3 + d2 * d2));
        }
        nextStep = fmax(1e-12, fmin(1e12, pow(accRel, 1. / 8) * sqrt(h2)));
    }

    /// one accepted step no longer than maxStep (> 0); returns its length, 0 on failure
    __device__ double step(double maxStep)
    {
        using namespace dp853;
        double h = fmin(maxStep, nextStep);
        int nbad = 0;
        double preverr = INFINITY;
        double k2[N], k3[N], k4[N], k5[N], k6[N], k7[N], k8[N], k9[N], k10[N], xt[N], k1b[N];
        for(int attempt = 0; attempt < 1000; attempt++) {
            if(h == 0 || !isFinite(h)) return 0;
            for(int i = 0; i < N; i++) xt[i] = x[i] + h * a21 * k1[i];
            f(xt, k2);
            for(int i = 0; i < N; i++) xt[i] = x[i] + h * (a31 * k1[i] + a32 * k2[i]);
            f(xt, k3);
            for(int i = 0; i < N; i++) xt[i] = x[i] + h * (a41 * k1[i] + a43 * k3[i]);
            f(xt, k4);
            for(int i = 0; i < N; i++) xt[i] = x[i] + h * (a51 * k1[i] + a53 * k3[i] + a54 * k4[i]);
            f(xt, k5);
            for(int i = 0; i < N; i++) xt[i] = x[i] + h * (a61 * k1[i] + a64 * k4[i] + a65 * k5[i]);
            f(xt, k6);
            for(int i = 0; i < N; i++) xt[i] = x[i] + h * (a71 * k1[i] + a74 * k4[i] + a75 * k5[i] + a76 * k6[i]);
            f(xt, k7);
            for(int i = 0; i < N; i++)
                xt[i] = x[i] + h * (a81 * k1[i] + a84 * k4[i] + a85 * k5[i] + a86 * k6[i] + a87 * k7[i]);
            f(xt, k8);
            for(int i = 0; i < N; i++)
                xt[i] = x[i] + h * (a91 * k1[i] + a94 * k4[i] + a95 * k5[i] + a96 * k6[i] + a97 * k7[i] + a98 * k8[i]);
            f(xt, k9);
            for(int i = 0; i < N; i++)
                xt[i] = x[i] + h * (a101 * k1[i] + a104 * k4[i] + a105 * k5[i] + a106 * k6[i] + a107 * k7[i] +
                    a108 * k8[i] + a109 * k9[i]);
            f(xt, k10);
            double* k11 = k2;   // k2, k3 are free after stage 5
            for(int i = 0; i < N; i++)
                xt[i] = x[i] + h * (a111 * k1[i] + a114 * k4[i] + a115 * k5[i] + a116 * k6[i] + a117 * k7[i] +
                    a118 * k8[i] + a119 * k9[i] + a1110 * k10[i]);
            f(xt, k11);
            double* k12 = k3;
            for(int i = 0; i < N; i++)
                xt[i] = x[i] + h * (a121 * k1[i] + a124 * k4[i] + a125 * k5[i] + a126 * k6[i] + a127 * k7[i] +
                    a128 * k8[i] + a129 * k9[i] + a1210 * k10[i] + a1211 * k11[i]);
            f(xt, k12);
            for(int i = 0; i < N; i++) {
                k1b[i] = b1 * k1[i] + b6 * k6[i] + b7 * k7[i] + b8 * k8[i] + b9 * k9[i] + b10 * k10[i] +
                    b11 * k11[i] + b12 * k12[i];
                xt[i] = x[i] + h * k1b[i];
            }
            double* k13 = k4;   // k4 is not needed after stage 12
            f(xt, k13);
            double err5 = 0, err3 = 0;
            for(int i = 0; i < N; i++) {
                const double sk = accRel * fmax(fabs(x[i]), fabs(xt[i]));
                if(sk == 0) continue;
                err3 += pow2((k1b[i] - bhh1 * k1[i] - bhh2 * k9[i] - bhh3 * k12[i]) / sk);
                err5 += pow2((er1 * k1[i] + er6 * k6[i] + er7 * k7[i] + er8 * k8[i] + er9 * k9[i] +
                    er10 * k10[i] + er11 * k11[i] + er12 * k12[i]) / sk);
            }
            const double den = sqrt(N * (err5 + 0.01 * err3));
            const double err = den == 0 ? 0 : err5 * fabs(h) / den;
            if(!isFinite(err)) return 0;
            double fac = sqrt(sqrt(sqrt(err)));
            bool accepted = false;
            if(err <= 1) {
                nextStep = fabs(h) * fmin(finc, safe / fac);
                accepted = true;
            } else {
                if(err > 0.5 * preverr) {
                    nbad++;
                    if(nbad >= 2) fac = 1 / fdec;
                    if(nbad >= 4) { nextStep = fabs(h); accepted = true; }
                } else
                    nbad = 0;
                if(!accepted) { preverr = err; h *= fmax(fdec, safe / fac); }
            }
            if(accepted) {
                for(int i = 0; i < N; i++) {
                    r[0][i] = x[i];
                    const double xd = xt[i] - x[i];
                    r[1][i] = xd;
                    const double xc = h * k1[i] - xd;
                    r[2][i] = xc;
                    r[3][i] = xd - h * k13[i] - xc;
                    r[4][i] = h * (d41 * k1[i] + d46 * k6[i] + d47 * k7[i] + d48 * k8[i] + d49 * k9[i] +
                        d410 * k10[i] + d411 * k11[i] + d412 * k12[i] + d413 * k13[i]);
                    r[5][i] = h * (d51 * k1[i] + d56 * k6[i] + d57 * k7[i] + d58 * k8[i] + d59 * k9[i] +
                        d510 * k10[i] + d511 * k11[i] + d512 * k12[i] + d513 * k13[i]);
                    r[6][i] = h * (d61 * k1[i] + d66 * k6[i] + d67 * k7[i] + d68 * k8[i] + d69 * k9[i] +
                        d610 * k10[i] + d611 * k11[i] + d612 * k12[i] + d613 * k13[i]);
                    r[7][i] = h * (d71 * k1[i] + d76 * k6[i] + d77 * k7[i] + d78 * k8[i] + d79 * k9[i] +
                        d710 * k10[i] + d711 * k11[i]);
                    x[i] = xt[i];
                    k1[i] = k13[i];
                }
                prevStep = h;
                return h;
            }
        }
        return 0;
    }

    /// dense output within the last step (OdeStepperDOP853::getSol, src/math_ode.cpp:409-426)
    __device__ double sol(double off, int i) const
    {
        if(off == prevStep) return x[i];
        if(off == 0) return r[0][i];
        const double p = off / prevStep, q = 1.0 - p;
        return r[0][i] + p * (r[1][i] + q * (r[2][i] + p * (r[3][i] + q * (r[4][i] + p * (r[5][i] +
            q * (r[6][i] + p * r[7][i]))))));
    }
};

/// z(t) within the last step and its derivative vz(t) (FindCrossingPointZequal0)
template<class Stepper>
struct CrossingFn {
    static constexpr bool hasDeriv = true;
    const Stepper* s;
    __device__ void operator()(double t, double* v, double* d) const {
        if(v) *v = s->sol(t, 1);
        if(d) *d = s->sol(t, 3);
    }
};

/** launch an orbit from (R0, z=0) with vz > 0 and find where it crosses z = 0 downward, with the
    derivative dRcross/dR0 from the variational equations (findCrossingPointR, :150-219) */
static __device__ void shellCrossing(const MultipoleView& M, double E, double Lz, double R0,
    double& Rcross, double& dRcrossdR0)
{
    double Phi;
    CylDerivs g; CylHess h;
    evalMultipoleCylCall<3, EVAL_AXI>(M, R0, 0, 0, &Phi, &g, &h);
    const double vz0 = sqrt(fmax(2 * (E - Phi) - (Lz > 0 ? pow2(Lz / R0) : 0), 0.));
    const double dR0 = 1.;
    const double dvz0 = vz0 > 0 ? ((Lz > 0 ? pow2(Lz) / (R0 * R0 * R0) : 0) - g.dR) / vz0 * dR0 : 0;
    const double vars[8] = { R0, 0, 0, vz0, dR0, 0, 0, dvz0 };
    MeridionalRHS rhs{ &M, Lz * Lz };
    Dop853Dense<8, MeridionalRHS> st{ rhs, SHELL_ACCURACY_INTEGR };
    st.init(vars);
    for(int n = 0; ; n++) {
        const double dt = st.step(INFINITY);
        if(dt <= 0 || n >= SHELL_MAX_NUM_STEPS_ODE) { Rcross = R0; dRcrossdR0 = NAN; return; }
        if(st.sol(dt, 1) <= 0) {
            CrossingFn<Dop853Dense<8, MeridionalRHS>> cf{ &st };
            const double tc = findRoot(cf, 0, dt, SHELL_ACCURACY_RSHELL);
            Rcross = st.sol(tc, 0);
            const double vR = st.sol(tc, 2), vz = st.sol(tc, 3), dR = st.sol(tc, 4), dz = st.sol(tc, 5);
            dRcrossdR0 = dR - dz * vR / vz;
            if(Rcross < 0) { Rcross = -Rcross; dRcrossdR0 = -dRcrossdR0; }
            return;
        }
    }
}

/// difference between the start and return radii of the orbit launched from R0 (FindClosedOrbitRZplane)
struct ClosedOrbitFn {
    static constexpr bool hasDeriv = true;
    const MultipoleView* M; double E, Lz, Rmin, Rmax;
    __device__ void operator()(double R0, double* val, double* der) const {
        if(R0 == Rmin || R0 == Rmax) {
            if(val) *val = R0 == Rmin ? Rmax - Rmin : Rmin - Rmax;
            if(der) *der = NAN;
            return;
        }
        double Rc, dRc = NAN;
        shellCrossing(*M, E, Lz, R0, Rc, dRc);
        if(val) *val = Rc - R0;
        if(der) *der = dRc - 1;
    }
};

/// focal distance of the shell orbit with energy E and angular momentum Lz; also its radius
/// (estimateFocalDistanceShellOrbit, :257-297, non-OLD_METHOD branch)
static __device__ double shellFocalDistance(const MultipoleView& M, double E, double Lz, double* Rshell)
{
    double Rmin, Rmax;
    shellPlanarExtent(M, E, Lz, Rmin, Rmax);
    ClosedOrbitFn f{ &M, E, Lz, Rmin, Rmax };
    const double Rsh = findRoot(f, Rmin, Rmax, SHELL_ACCURACY_RSHELL);
    double Phi;
    CylDerivs g; CylHess h;
    evalMultipoleCylCall<3, EVAL_AXI>(M, Rsh, 0, 0, &Phi, &g, &h);
    const double vphi = Lz != 0 ? Lz / Rsh : 0;
    const double FD = Rsh * sqrt(clip((2 * (E - Phi) - Rsh * g.dR) / (Rsh * g.dR - vphi * vphi), 0., 1e6));
    if(Rshell) *Rshell = Rsh;
    return FD;
}

}  // namespace agb
