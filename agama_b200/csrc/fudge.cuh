// Axisymmetric Staeckel-fudge actions on the device (one phase-space point per thread).
//
// Reference: src/actions_staeckel.cpp -- findIntegralsOfMotionAxisymFudge (:176-195),
// AxisymFunctionFudge::evalDeriv (:202-252), AxisymIntegrand (:276-299),
// AxisymScaledForRootfinder (:329-354), findIntegrationLimitsAxisym (:360-483),
// computeActions (:604-619), evalAxisym (:645-670), evalAxisymFudge (:683-693) and
// ActionFinderAxisymFudge::eval (:954-979); prolate spheroidal coordinates from src/coord.cpp
// (:266-338, :525-531); L_circ(E) from potential::Interpolator (src/potential_utils.cpp:872-980).
#pragma once
#include "multipole_eval.cuh"
#include "fudge_types.h"

namespace agb {

constexpr int FUDGE_INTEGR_ORDER = 10;           // src/actions_staeckel.cpp:21
constexpr double FUDGE_ACCURACY_RANGE = 1e-6;    // src/actions_staeckel.cpp:35
constexpr double FUDGE_MINIMUM_RANGE = 1e-10;    // src/actions_staeckel.cpp:38

/// QuinticSpline::evalDeriv (src/math_spline.cpp:1405-1429): linear extrapolation outside
__device__ __forceinline__ void spline1d(const Spline1dView& S, double x, double* f, double* df, double* d2f)
{
    const int n = S.n;
    const double* xv = S.t;
    const double* fv = S.t + n;
    const double* f1 = S.t + 2 * n;
    const double* f2 = S.t + 3 * n;
    if(n == 0 || x != x) { *f = NAN; if(df) *df = NAN; if(d2f) *d2f = NAN; return; }
    const int i = binSearch(x, xv, n);
    if(i < 0 || i >= n - 1) {
        const int e = i < 0 ? 0 : n - 1;
        const double d = ldg(f1 + e);
        *f = ldg(fv + e) + (d == 0 ? 0 : d * (x - ldg(xv + e)));
        if(df) *df = d;
        if(d2f) *d2f = 0;
        return;
    }
    const double fl[1] = { ldg(fv + i) }, fh[1] = { ldg(fv + i + 1) }, d1l[1] = { ldg(f1 + i) },
        d1h[1] = { ldg(f1 + i + 1) }, d2l[1] = { ldg(f2 + i) }, d2h[1] = { ldg(f2 + i + 1) };
    quinticSegment<1>(x, ldg(xv + i), ldg(xv + i + 1), fl, fh, d1l, d1h, d2l, d2h, f, df, d2f);
}

/// potential::Interpolator::evalDeriv (src/potential_utils.cpp:872-911): Phi(R), dPhi/dR, d2Phi/dR2
static __device__ void interpPhi(const FudgeTables& F, double R, double* val, double* der, double* der2)
{
    const double logR = log(R);
    if(logR > ldg(F.PhiofR.t + F.PhiofR.n - 1) && F.coefOut != 0) {
        const double Rs = exp(logR * F.slopeOut);
        const double Phi = (-F.massOut + (F.slopeOut == -1 ? logR : (R * Rs - 1) / (F.slopeOut + 1)) * F.coefOut) / R;
        *val = Phi;
        *der = (-Phi + F.coefOut * Rs) / R;
        *der2 = (2 * Phi + F.coefOut * Rs * (F.slopeOut - 2)) / pow2(R);
        return;
    }
    double s, d1, d2;
    spline1d(F.PhiofR, logR, &s, &d1, &d2);
    const double ex = exp(s), E = 1 / (F.iInvPhi0 - ex), dE = E * E * ex, d2E = E * dE * (F.iInvPhi0 + ex);
    *val = E;
    *der = dE * d1 / R;
    *der2 = (dE * (d2 - d1) + d2E * d1 * d1) / pow2(R);
}

/// potential::Interpolator::L_circ (src/potential_utils.cpp:954-980)
static __device__ double interpLcirc(const FudgeTables& F, double E)
{
    if(!(E >= 1. / F.iInvPhi0 && E <= 0))
        return NAN;
    const double scaledE = log(F.iInvPhi0 - 1 / E);
    double logL;
    spline1d(F.LofE, scaledE, &logL, nullptr, nullptr);
    double Lcirc = exp(logL);
    if(scaledE > ldg(F.LofE.t + F.LofE.n - 1)) {   // large-radius correction
        double logR;
        spline1d(F.RofL, logL, &logR, nullptr, nullptr);
        const double Rc = exp(logR);
        double Phi, dPhi, d2Phi;
        interpPhi(F, Rc, &Phi, &dPhi, &d2Phi);
        const double Ec = Phi + 0.5 * Rc * dPhi;
        const double denom = 1 - 0.5 * (Ec - E) * (Rc * d2Phi - dPhi) / ((Rc * d2Phi + 3 * dPhi) * Rc * dPhi);
        Lcirc = clip(sqrt(Rc * dPhi) * (Rc - (Ec - E) / (dPhi * denom)), 0.75 * Lcirc, 1.25 * Lcirc);
    }
    return Lcirc;
}

/// bilinear Delta(xi, chi) (LinearInterpolator2d::evalDeriv, src/math_spline.cpp:2152-2190)
static __device__ double deltaLookup(const FudgeTables& F, double x, double y)
{
    const int nx = F.nE, ny = F.nL;
    const int xi = binSearch(x, F.gridE, nx), yi = binSearch(y, F.gridL, ny);
    if(xi < 0 || xi >= nx - 1 || yi < 0 || yi >= ny - 1)
        return NAN;
    const double* f = F.delta + static_cast<size_t>(xi) * ny + yi;
    const double zll = ldg(f), zlu = ldg(f + 1), zul = ldg(f + ny), zuu = ldg(f + ny + 1);
    const double xl = ldg(F.gridE + xi), yl = ldg(F.gridL + yi);
    const double t = (x - xl) / (ldg(F.gridE + xi + 1) - xl), u = (y - yl) / (ldg(F.gridL + yi + 1) - yl);
    const double T = 1 - t, U = 1 - u;
    return T * (U * zll + u * zlu) + t * (U * zul + u * zuu);
}

/// the fudge's auxiliary function F(tau) and the integrals of motion of one point
struct FudgeFunction {
    const MultipoleView* M;
    double lambda, nu, phi, D2;     // point in prolate spheroidal coordinates (Delta^2 = D2)
    double E, Lz, I3, flambda, fnu;
    double Ilam, Inu, L2h;          // I3 - fnu, I3 - flambda and Lz^2 / 2, formed once (derive())
    int bad;                        // set when a coordinate conversion is invalid

    /// the terms of F that do not depend on tau, from the integrals of motion (the same
    /// operations as in F itself, so the same bits)
    __device__ void derive() { Ilam = I3 - fnu; Inu = I3 - flambda; L2h = Lz * Lz / 2; }

    /// F(tau) and optionally F', F'' (src/actions_staeckel.cpp:202-252); INL: the potential
    /// evaluation inlined at this call site instead of the shared out-of-line copy
    template<bool DER, bool DER2, bool INL = false>
    __device__ void eval(double tau, double* val, double* der, double* der2) const
    {
        double lam, n, mult, I;
        if(tau >= D2) { lam = tau; n = fabs(nu); mult = lam - n; I = Ilam; }
        else          { lam = lambda; n = tau; mult = n - lam; I = Inu; }
        // prolate spheroidal -> cylindrical (src/coord.cpp:266-291)
        const double absnu = fabs(n), sgn = n >= 0 ? 1 : -1;
        const double lmd = lam - D2, nmd = absnu - D2;
        if(nmd > 0 || lmd < 0) {
            *val = NAN; if(DER) *der = NAN; if(DER2) *der2 = NAN;
            return;
        }
        const double R = sqrt(lmd * (1 - absnu / D2));
        const double z = sqrt(lam * absnu / D2) * sgn;
        double Phi;
        CylDerivs g; CylHess h;
        // the inlined F, F' of the root searches: the cell evaluated in halves (fewer registers
        // beside the searches' state, the same bits)
        if(INL)      evalMultipoleCyl<DER2 ? 6 : DER ? 3 : 1, EVAL_AXI, 1, false, DER && !DER2>(*M, R, z, phi, &Phi, &g, &h);
        else if(DER2) evalMultipoleCylCall<6, EVAL_AXI>(*M, R, z, phi, &Phi, &g, &h);
        else if(DER) evalMultipoleCylCall<3, EVAL_AXI>(*M, R, z, phi, &Phi, &g, &h);
        else         evalMultipoleCylCall<1, EVAL_AXI>(*M, R, z, phi, &Phi, &g, &h);
        const double tmd = tau - D2;
        *val = (tmd != 0 ? (E * tau - I - Phi * mult) * tmd : 0) - L2h * tau;
        if(DER || DER2) {
            // dR/dtau, dz/dtau along the coordinate that tau moves (lambda or nu): only that pair
            // is divided out
            const bool lbranch = tau >= D2;
            double dRdt, dzdt;
            if(lbranch) { dRdt = 0.5 * R / lmd; dzdt = 0.5 * z / lam; }
            else        { dRdt = 0.5 * R / nmd * sgn; dzdt = 0.5 * z / n; }
            const double dPhidtau = g.dR * dRdt + g.dz * dzdt;
            if(DER)
                *der = E * (tau + tmd) - L2h - I - (mult + tmd) * Phi -
                       (tmd != 0 ? tmd * mult * dPhidtau : 0);
            if(DER2) {
                double d2;
                if(lbranch) {
                    const double d2Rdl2 = -0.25 * R / pow2(lmd), d2zdl2 = -0.25 * z / pow2(lam);
                    d2 = h.dR2 * pow2(dRdt) + h.dz2 * pow2(dzdt) + 2 * h.dRdz * dRdt * dzdt +
                         g.dR * d2Rdl2 + g.dz * d2zdl2;
                } else {
                    const double d2Rdn2 = -0.25 * R / pow2(nmd), d2zdn2 = -0.25 * z / pow2(n);
                    d2 = h.dR2 * pow2(dRdt) + h.dz2 * pow2(dzdt) + 2 * h.dRdz * dRdt * dzdt +
                         g.dR * d2Rdn2 + g.dz * d2zdn2;
                }
                *der2 = 2 * (E - Phi - (mult + tmd) * dPhidtau) - tmd * mult * d2;
            }
        }
    }
    __device__ double value(double tau) const { double v; eval<false, false, true>(tau, &v, nullptr, nullptr); return v; }
};

/// State of one point between the phases of the action computation: the point in prolate
/// spheroidal coordinates, its integrals of motion, the integration limits known so far and the
/// brackets of the roots still to be found.  One 128-byte record per point.
struct __align__(16) FudgeRecord {
    double lambda, nu, D2, E, Lz, I3, flambda, fnu, phi;
    double lambdaMin, lambdaMax, nuMax;     // nu_min is always 0
    double nuUpper;                         // nu_max root bracket: [|nu|, nuUpper]
    double lambdaLower, lambdaPos;          // lambda_min root in [lambdaLower, lambdaPos];
                                            // lambda_max root in [lambdaPos, inf)
    int roots;                              // ROOT_* bits of the roots still to be found
    int valid;                              // 0: the point has no integrals to do; otherwise
                                            // REC_VALID | the REC_* direction-of-motion bits
};

/// bits of FudgeRecord::valid: the point has integrals to do, and the signs of its motion in
/// prolate spheroidal coordinates that the angles need (lambdadot >= 0, nudot * nu >= 0, nudot < 0)
enum { REC_VALID = 1, REC_LDOT_POS = 2, REC_NDOT_NU_POS = 4, REC_NUDOT_NEG = 8 };
static_assert(sizeof(FudgeRecord) == 128, "FudgeRecord is one 128-byte line");

enum { ROOT_NU_MAX = 1, ROOT_LAMBDA_MIN = 2, ROOT_LAMBDA_MAX = 4 };

/// F and F' at the ends of the plain root brackets that phase 1 evaluates once for the searches of
/// phase 2: lambda_pos (shared by the lambda_min and lambda_max brackets), Delta^2 (the upper end
/// of the nu_max bracket and the lower end of the lambda_min one) and |nu| (the lower end of the
/// nu_max bracket); NaN where not evaluated
struct FudgeEnds { double fPos, dfPos, fD2, dfD2, fNu, dfNu; };

/** The root functions of the three integration limits behind one evaluation site (kind
    ROOT_NU_MAX, ROOT_LAMBDA_MIN: F(tau) and F'(tau); ROOT_LAMBDA_MAX: F(tau)/tau^2 on
    [u0, inf) mapped to s in [0, 1] by the semi-infinite scaling, AxisymScaledForRootfinder inside
    ScaledFnc<ScalingSemiInf>, src/actions_staeckel.cpp:329-354, src/math_core.h:214-232). */
__device__ __forceinline__ void limitRootEval(const FudgeFunction& f, int kind, double u0, double x,
    double* v, double* d)
{
    const bool semiInf = kind == ROOT_LAMBDA_MAX;
    double duds = 1, tau = x;
    if(semiInf) tau = unscaleSemiInf(u0, x, &duds);
    const bool far = semiInf && tau > 1e100;
    double fval = 0, fder = 0;
    if(!far) f.eval<true, false, true>(tau, &fval, &fder, nullptr);
    if(!semiInf) { *v = fval; *d = fder; }
    else if(far) { *v = f.E; *d = NAN; }
    else {
        *v = fval / pow2(tau);
        *d = (fder - 2 * fval / tau) / pow2(tau) * duds;
    }
}

/** The point's F(tau) from its record.  The azimuth given to the potential is 0: the fudge takes
    only axisymmetric potentials, whose coefficients (and so the index sets of their splines and
    asymptotes) have m = 0 alone, and their evaluators never read the azimuth; a constant leaves
    the register free for the searches (the record keeps the point's azimuth for the angles). */
__device__ __forceinline__ void loadFudgeFunction(const MultipoleView& M, const FudgeRecord& r, FudgeFunction& f)
{
    f.M = &M;
    f.lambda = r.lambda; f.nu = r.nu; f.phi = 0; f.D2 = r.D2;
    f.E = r.E; f.Lz = r.Lz; f.I3 = r.I3; f.flambda = r.flambda; f.fnu = r.fnu;
    f.derive();
    f.bad = 0;
}

/** Integration limits of the lambda and nu motions (findIntegrationLimitsAxisym,
    src/actions_staeckel.cpp:360-483), part 1: every decision up to the three root searches, whose
    brackets go into the record; limits that need no root are stored directly (NaN otherwise).
    ends (may be null) receives F and F' at the ends of the plain brackets (FudgeEnds), which the
    root searches then take instead of evaluating them: at lambda_pos from the evaluation above,
    at Delta^2 and |nu| from the same evaluation of F as the searches would make. */
static __device__ void fudgeLimitsSetup(const FudgeFunction& fnc, FudgeRecord& rec, FudgeEnds* ends = nullptr)
{
    const double delta = fnc.D2;
    const double f_zero = fnc.value(0);
    double f_lambda, df_lambda, d2f_lambda;
    fnc.eval<true, true>(fnc.lambda, &f_lambda, &df_lambda, &d2f_lambda);
    double nu_max = NAN, lambda_min = NAN, lambda_max = NAN;
    double nu_upper = delta, lambda_lower = delta;
    int roots = 0;
    if(fnc.Lz == 0) {
        const double dminus = delta * (1 - 1e-15), dplus = delta * (1 + 1e-15);
        if(fnc.value(dminus) < 0) {
            if(f_zero > 0) nu_upper = dminus;
            else nu_max = 0;
        } else
            nu_max = delta;
        if(fnc.value(dplus) < 0) lambda_lower = dplus;
        else lambda_min = delta;
    }
    if(!isFinite(nu_max)) {
        if(f_zero > 0) roots |= ROOT_NU_MAX;           // falls back to |nu| if no root is found
        else nu_max = fabs(fnc.nu);
    }
    double lambda_pos = fnc.lambda, f_pos = f_lambda, df_pos = df_lambda;
    const double dxToRoot = -f_lambda / df_lambda;
    if(f_lambda <= 0 || fabs(dxToRoot) < fnc.lambda * FUDGE_MINIMUM_RANGE) {
        if(df_lambda >= 0) lambda_min = fnc.lambda;
        if(df_lambda <= 0) {
            lambda_max = fnc.lambda;
            if(fnc.lambda == delta) lambda_min = delta;
        }
        bool nearShell = d2f_lambda < 0 &&
            pow2(df_lambda) - 2 * f_lambda * d2f_lambda - pow2(fnc.lambda * FUDGE_MINIMUM_RANGE * d2f_lambda) < 0;
        const double safeOffset = fmin(0.5 * fabs(df_lambda / d2f_lambda), fnc.lambda * FUDGE_MINIMUM_RANGE);
        lambda_pos += fmax(dxToRoot, safeOffset) * (df_lambda >= 0 ? 1 : -1);
        double f_lp, df_lp, d2f_lp;
        fnc.eval<true, true>(lambda_pos, &f_lp, &df_lp, &d2f_lp);
        f_pos = f_lp; df_pos = df_lp;
        nearShell |= d2f_lp < 0 &&
            pow2(df_lp) - 2 * f_lp * d2f_lp - pow2(fnc.lambda * FUDGE_MINIMUM_RANGE * d2f_lp) < 0;
        if(nearShell || f_lp < 0)
            lambda_min = lambda_max = fnc.lambda;
    }
    if(!isFinite(lambda_min)) roots |= ROOT_LAMBDA_MIN;
    if(!isFinite(lambda_max)) roots |= ROOT_LAMBDA_MAX;
    rec.nuMax = nu_max; rec.lambdaMin = lambda_min; rec.lambdaMax = lambda_max;
    rec.nuUpper = nu_upper; rec.lambdaLower = lambda_lower; rec.lambdaPos = lambda_pos;
    rec.roots = roots;
    if(ends) {
        ends->fPos = f_pos; ends->dfPos = df_pos;
        ends->fD2 = ends->dfD2 = ends->fNu = ends->dfNu = NAN;
        if(((roots & ROOT_NU_MAX) && nu_upper == delta) || ((roots & ROOT_LAMBDA_MIN) && lambda_lower == delta))
            fnc.eval<true, false>(delta, &ends->fD2, &ends->dfD2, nullptr);
        if(roots & ROOT_NU_MAX)
            fnc.eval<true, false>(fabs(fnc.nu), &ends->fNu, &ends->dfNu, nullptr);
    }
}

struct FudgeLimits { double lambda_min, lambda_max, nu_max; int order; };

/** Part 3 (part 2 is the root searches: RootSearch driven by limitRootEval): the final checks of
    the limits and the Gauss-Legendre order of both integrals. */
static __device__ FudgeLimits fudgeLimitsFinish(const FudgeRecord& rec)
{
    const double delta = rec.D2;
    FudgeLimits lim{ rec.lambdaMin, rec.lambdaMax, rec.nuMax, 0 };
    if(!(lim.nu_max >= delta * FUDGE_MINIMUM_RANGE))
        lim.nu_max = 0;
    if(!(lim.lambda_max - lim.lambda_min >= delta * FUDGE_MINIMUM_RANGE))
        lim.lambda_min = lim.lambda_max = rec.lambda;
    const double ratio = sqrt((lim.lambda_min - delta) / (lim.lambda_max - delta));
    if(ratio == 0) lim.order = GL_MAX_ORDER;
    else {
        int e;
        frexp(ratio, &e);
        lim.order = min(GL_MAX_ORDER, FUDGE_INTEGR_ORDER - e);
    }
    return lim;
}

/** One node of the momentum integral of sqrt(p^2(tau)) over [lo, hi] with the cubic end-point
    stretch (integrateGL of ScaledIntegrand<ScalingCub>(AxisymIntegrand), src/math_core.cpp:1191-1205,
    src/actions_staeckel.cpp:276-299): the integrand times du/ds at the scaled node s. */
static __device__ double fudgeMomentumNode(const FudgeFunction& fnc, double lo, double hi, double s)
{
    double duds;
    const double tau = unscaleCub(lo, hi, s, &duds);
    const double tmd = tau - fnc.D2;
    const double p2 = fnc.value(tau) / (2 * pow2(tmd) * tau);
    double v = p2 < 0 ? 0 : sqrt(p2);
    if(!isFinite(v)) v = 0;
    return v * duds;
}

/** The same node with the integrand's arithmetic in FP32 (the mixed-precision form of the action
    quadrature): F(tau) and the point tau come from FP64 (the potential and the cancellation in
    F stay FP64), then p = sqrt(F / (2 tau)) / |tau - D2| (the square root through the hardware
    reciprocal square root) and the product with du/ds are FP32; the caller accumulates the weighted
    terms with compensation. */
static __device__ float fudgeMomentumNode32(const FudgeFunction& fnc, double lo, double hi, double s)
{
    double duds;
    const double tau = unscaleCub(lo, hi, s, &duds);
    const double F = fnc.value(tau);
    // p = sqrt(F / (2 tau)) / |tau - D2|: the square root before the division by (tau - D2)^2
    // keeps every FP32 intermediate in range for tau up to ~1e18 (the product (tau - D2)^2 tau
    // overflows FP32 already at tau ~ 1e12, where loosely bound orbits reach); a value of F
    // beyond the FP32 range takes the FP64 form
    if(!(fabs(F) < 1e37)) return static_cast<float>(fudgeMomentumNode(fnc, lo, hi, s));
    const float tmd = static_cast<float>(tau - fnc.D2), t = static_cast<float>(tau);
    const float q = static_cast<float>(F) / (2.f * t);
    float v = q > 0.f ? q * rsqrtf(q) / fabsf(tmd) : 0.f;
    if(!(v < INFINITY)) v = 0.f;
    return v * static_cast<float>(duds);
}

/** Phase 1 of the actions of one point (R, z, phi, vR, vz, vphi) for focal distance fd
    (evalAxisymFudge, src/actions_staeckel.cpp:683-693: fd <= 0 falls back to max(R,1)*1e-4);
    Phi is the potential at the point.  Writes Jphi into act[2]; for a point without actions
    (unbound, or lambda = nu = Delta^2) also NaN into act[0..1] and marks the record invalid.
    Otherwise the record holds the integrals of motion (findIntegralsOfMotionAxisymFudge,
    :176-195) and the limits and root brackets of fudgeLimitsSetup (ends: as there). */
static __device__ void fudgePrepare(const MultipoleView& M, const double* pc, double Phi, double fd,
    FudgeRecord& rec, double* act, FudgeEnds* ends = nullptr)
{
    const double R = pc[0], z = pc[1], phi = pc[2], vR = pc[3], vz = pc[4], vphi = pc[5];
    if(fd <= 0) fd = fmax(R, 1.) * 1e-4;
    const double D2 = fd * fd;
    const double Lz = R * vphi;
    act[2] = Lz;
    rec.valid = 0;
    rec.roots = 0;
    // cylindrical -> prolate spheroidal (src/coord.cpp:294-338) and velocities (:525-531)
    const double R2 = R * R, z2 = z * z, signz = z >= 0 ? 1 : -1;
    const double sum = R2 + z2 + D2, dif = R2 + z2 - D2;
    double sqD = sqrt(pow2(dif) + 4 * R2 * D2);
    if(z2 == 0) sqD = sum;
    if(R2 == 0) sqD = fabs(dif);
    double lmd, dmn;
    if(dif >= 0) { lmd = 0.5 * (sqD + dif); dmn = R2 > 0 ? D2 * R2 / lmd : 0; }
    else         { dmn = 0.5 * (sqD - dif); lmd = D2 * R2 / dmn; }
    const double lambda = D2 + lmd;
    double absnu = 2 * D2 / (sum + sqD) * z2;
    if(absnu * 2 > D2) absnu = D2 - dmn; else dmn = D2 - absnu;
    if(sqD == 0) { act[0] = act[1] = NAN; return; }   // lambda = nu = Delta^2: undefined
    FudgeFunction fnc;
    fnc.M = &M;
    fnc.lambda = lambda;
    fnc.nu = absnu * signz;
    fnc.phi = 0;                    // axisymmetric potential: its evaluators never read the azimuth
    fnc.D2 = D2;
    fnc.bad = 0;
    double Phi0;
    CylDerivs g; CylHess h;
    evalMultipoleCylCall<1, EVAL_AXI>(M, sqrt(lambda - D2), 0, 0, &Phi0, &g, &h);
    const double Ekin = 0.5 * (vR * vR + vz * vz + vphi * vphi);
    fnc.E = Phi + Ekin;
    fnc.Lz = Lz;
    fnc.flambda = -lambda * Phi0;
    fnc.fnu = fnc.flambda + Phi * (lambda - absnu);
    fnc.I3 = lambda * (Phi - Phi0) + 0.5 * (pow2(z * vphi) + pow2(R * vz - z * vR) + pow2(vz) * D2);
    fnc.derive();
    if(!isFinite(fnc.E + fnc.I3 + fnc.Lz) || fnc.E >= 0) { act[0] = act[1] = NAN; return; }
    rec.lambda = fnc.lambda; rec.nu = fnc.nu; rec.D2 = D2; rec.E = fnc.E; rec.Lz = Lz; rec.I3 = fnc.I3;
    rec.flambda = fnc.flambda; rec.fnu = fnc.fnu; rec.phi = phi;
    fudgeLimitsSetup(fnc, rec, ends);
    // velocities in prolate spheroidal coordinates (src/coord.cpp:317-322, :525-531)
    const double lambdadot = R * 2 * lambda / sqD * vR + z * 2 * lmd / sqD * vz;
    const double nudot = R * 2 * -absnu / sqD * signz * vR + z * 2 * dmn / sqD * signz * vz;
    rec.valid = REC_VALID | (lambdadot >= 0 ? REC_LDOT_POS : 0) | (nudot * fnc.nu >= 0 ? REC_NDOT_NU_POS : 0) |
        (nudot < 0 ? REC_NUDOT_NEG : 0);
}

/** Inverse of the cubic end-point scaling (math::scale of ScalingCub, src/math_core.cpp:370-386):
    s in [0, 1] with u = ul (1-s)^2 (1+2s) + ur s^2 (3-2s).  On the nearer half, w = s^2 (3 - 2s) is
    a depressed cubic in y = s - 1/2 whose trigonometric root s = 1/2 + cos((acos(1 - 2w) - 2pi)/3)
    is polished by three Newton steps; u outside [ul, ur] gives NaN, as in the reference. */
static __device__ double scaleCubInverse(double ul, double ur, double u)
{
    if(u == ul) return 0;
    if(u == ur) return 1;
    const double half = 0.5 * (ul + ur);
    if(u == half) return 0.5;
    const double w = u < half ? (u - ul) / (ur - ul) : (ur - u) / (ur - ul);
    double s = 0.5 + cos((acos(1 - 2 * w) - 2 * M_PI) / 3);
    for(int i = 0; i < 3; i++)
        s -= (s * s * (3 - 2 * s) - w) / (6 * s * (1 - s));
    return u < half ? s : 1 - s;
}

/// the three integrands of AxisymIntegrand::value with p in the denominator (n = -1), from one
/// F(tau): (tau-Delta^2)^-1 [E], (tau-Delta^2)^-1 tau^-1 [I3], (tau-Delta^2)^-2 with the singular
/// part at nu_max removed [Lz] (src/actions_staeckel.cpp:276-299)
struct InverseMomentumTerms { double e, i3, lz; };

static __device__ InverseMomentumTerms inverseMomentumTerms(double ft, double tau, double D2, double nuMax,
    double dfdnuMax)
{
    InverseMomentumTerms t{ 0, 0, 0 };
    const double tmd = tau - D2;
    const double p2 = ft / (2 * pow2(tmd) * tau);
    if(p2 < 0) return t;
    const double r = 1 / sqrt(p2);
    double v = r / tmd;
    t.e = isFinite(v) ? v : 0;
    v = r / tmd / tau;
    t.i3 = isFinite(v) ? v : 0;
    v = r / pow2(tmd);
    if(tmd < 0) v += sqrt(2 * nuMax / dfdnuMax / (tau - nuMax)) / tmd;
    t.lz = isFinite(v) ? v : 0;
    return t;
}

/// GL rule of the requested order (the next tabulated one at or above it)
static __device__ __forceinline__ int glRule(const GLRules& gl, int order, const double** x, const double** w)
{
    int N = order < 1 ? 1 : order;
    while(gl.offset[N] < 0) N++;
    *x = gl.nodes + gl.offset[N];
    *w = gl.weights + gl.offset[N];
    return N;
}

/** the inverse-momentum integrals of one branch over the scaled interval [0, y] of [lo, hi]
    (integrateGL(ScaledIntegrand<ScalingCub>, 0, y, N), src/math_core.cpp:1191-1205); with
    ACT also the action integral (p in the numerator) over the same nodes, when y = 1 */
template<bool ACT>
static __device__ InverseMomentumTerms branchIntegrals(const FudgeFunction& fnc, const GLRules& gl, int order,
    double lo, double hi, double y, double nuMax, double dfdnuMax, double* act)
{
    InverseMomentumTerms sum{ 0, 0, 0 };
    if(ACT) *act = 0;
    if(y == 0) return sum;
    const double *x, *w;
    const int N = glRule(gl, order, &x, &w);
    double sa = 0;
    for(int i = 0; i < N; i++) {
        const double xi = ldg(x + i), wi = ldg(w + i);
        double duds;
        const double tau = unscaleCub(lo, hi, y * xi + 0 * (1 - xi), &duds);
        const double ft = fnc.value(tau);
        const InverseMomentumTerms t = inverseMomentumTerms(ft, tau, fnc.D2, nuMax, dfdnuMax);
        sum.e += wi * (t.e * duds);
        sum.i3 += wi * (t.i3 * duds);
        sum.lz += wi * (t.lz * duds);
        if(ACT) {
            const double tmd = tau - fnc.D2;
            const double p2 = ft / (2 * pow2(tmd) * tau);
            double v = p2 < 0 ? 0 : sqrt(p2);
            if(!isFinite(v)) v = 0;
            sa += wi * (v * duds);
        }
    }
    sum.e *= y; sum.i3 *= y; sum.lz *= y;
    if(ACT) *act = sa * y;
    return sum;
}

/// 2 pi wrap of an angle into [0, 2 pi) (math::wrapAngle, src/math_core.cpp:149-157; NaN -> 0)
static __device__ __forceinline__ double wrapAngle(double x)
{
    x -= 2 * M_PI * floor(1 / (2 * M_PI) * x);
    return x >= 0 && x < 2 * M_PI ? x : 0;
}

/** Actions, frequencies and angles of a prepared point whose roots are found (evalAxisym,
    src/actions_staeckel.cpp:645-670): computeActions (:604-619), computeActionDerivatives
    (:489-527), computeIntDerivatives (:532-560), computeGenFuncDerivatives (:566-600) and
    computeAngles (:624-636).  The action integrals and the derivative integrals share their
    potential evaluations (same nodes); ang / freq may be null. */
static __device__ void fudgeAnglesFrequencies(const MultipoleView& M, const GLRules& gl, const FudgeRecord& rec,
    double* act, double* ang, double* freq)
{
    FudgeFunction fnc;
    loadFudgeFunction(M, rec, fnc);
    const FudgeLimits lim = fudgeLimitsFinish(rec);
    const double D2 = rec.D2, Lz = rec.Lz;
    double dfdnuMax, unused;
    fnc.eval<true, false>(lim.nu_max, &unused, &dfdnuMax, nullptr);
    // action derivatives over (E, I3, Lz), full ranges; the actions from the same nodes
    double Jr, Jz;
    InverseMomentumTerms L = branchIntegrals<true>(fnc, gl, lim.order, lim.lambda_min, lim.lambda_max, 1,
        lim.nu_max, dfdnuMax, &Jr);
    const InverseMomentumTerms N = branchIntegrals<true>(fnc, gl, lim.order, 0, lim.nu_max, 1,
        lim.nu_max, dfdnuMax, &Jz);
    act[0] = Jr / M_PI;
    act[1] = Jz / M_PI * 2;
    if(lim.lambda_min == lim.lambda_max) {      // limitingIntegralValue, :307-323
        const double tau = lim.lambda_min, tmd = tau - D2;
        double d2, v0;
        fnc.eval<false, true>(tau, &v0, nullptr, &d2);
        const double base = 2 * M_PI * sqrt(-tau / d2) * fabs(tmd);
        L.e = base / tmd;
        L.i3 = base / tmd / tau;
        L.lz = base / pow2(tmd);
    }
    const double dJrdE = L.e / (4 * M_PI), dJzdE = N.e / (2 * M_PI);
    const double dJrdI3 = -L.i3 / (4 * M_PI), dJzdI3 = -N.i3 / (2 * M_PI);
    const double dJrdLz = -Lz * L.lz / (4 * M_PI);
    const double dmn = D2 - lim.nu_max;
    const double singpart = 2 * sqrt(-2 * lim.nu_max / dfdnuMax / dmn) * atan(sqrt(lim.nu_max / dmn));
    const double dJzdLz = -Lz * (N.lz + singpart) / (2 * M_PI);
    // inverse matrix: frequencies and the derivatives of I3 over the actions
    double Or, Oz, Ophi, dI3dJr, dI3dJz, dI3dJphi;
    const double det = dJrdE * dJzdI3 - dJrdI3 * dJzdE;
    if(lim.nu_max == 0 || det == 0) {
        Or = 1 / dJrdE;
        Ophi = -dJrdLz / dJrdE;
        dI3dJr = dI3dJz = dI3dJphi = Oz = 0;
    } else {
        Or = dJzdI3 / det;
        Oz = -dJrdI3 / det;
        Ophi = (dJrdI3 * dJzdLz - dJrdLz * dJzdI3) / det;
        dI3dJr = -dJzdE / det;
        dI3dJz = dJrdE / det;
        dI3dJphi = -(dJrdE * dJzdLz - dJrdLz * dJzdE) / det;
    }
    if(freq) { freq[0] = Or; freq[1] = Oz; freq[2] = Ophi; }
    if(!ang) return;
    // derivatives of the generating function over (E, I3, Lz): integrals up to the point
    const double signl = rec.valid & REC_LDOT_POS ? 1 : -1, signn = rec.valid & REC_NDOT_NU_POS ? 1 : -1;
    const double absnu = fabs(rec.nu);
    const double yl = scaleCubInverse(lim.lambda_min, lim.lambda_max, rec.lambda);
    const double yn = lim.nu_max == 0 ? 0 : scaleCubInverse(0, lim.nu_max, absnu);
    const InverseMomentumTerms Lp = branchIntegrals<false>(fnc, gl, lim.order, lim.lambda_min, lim.lambda_max, yl,
        lim.nu_max, dfdnuMax, nullptr);
    const InverseMomentumTerms Np = branchIntegrals<false>(fnc, gl, lim.order, 0, lim.nu_max, yn,
        lim.nu_max, dfdnuMax, nullptr);
    const double dSdE = signl * Lp.e / 4 + signn * Np.e / 4;
    const double dSdI3 = signl * -Lp.i3 / 4 + signn * -Np.i3 / 4;
    const double singS = 2 * sqrt(-2 * lim.nu_max / dfdnuMax / dmn) *
        (atan(sqrt(lim.nu_max / dmn)) - atan(sqrt((lim.nu_max - absnu) / dmn)));
    const double dSdLz = Lz == 0 ? 0 : rec.phi + signl * -Lz * Lp.lz / 4 + signn * -Lz * (Np.lz + singS) / 4;
    const bool addPi = (rec.valid & REC_NUDOT_NEG) && Lz != 0;
    ang[0] = wrapAngle(dSdE * Or + dSdI3 * dI3dJr + dSdLz * 0);
    ang[1] = wrapAngle(dSdE * Oz + dSdI3 * dI3dJz + dSdLz * 0 + M_PI * addPi);
    ang[2] = wrapAngle(dSdE * Ophi + dSdI3 * dI3dJphi + dSdLz * 1);
}

/// Cartesian posvel -> cylindrical (R, z, phi, vR, vz, vphi); reference src/coord.cpp:476-484
__device__ __forceinline__ void carToCylPosVel(const double* w, double* pc)
{
    const double R = sqrt(w[0] * w[0] + w[1] * w[1]);
    if(R == 0) {
        pc[0] = 0; pc[1] = w[2]; pc[2] = atan2(w[4], w[3]);
        pc[3] = sqrt(w[3] * w[3] + w[4] * w[4]); pc[4] = w[5]; pc[5] = 0;
        return;
    }
    const double c = w[0] / R, s = w[1] / R;
    pc[0] = R; pc[1] = w[2]; pc[2] = atan2(w[1], w[0]);
    pc[3] = w[3] * c + w[4] * s;
    pc[4] = w[5];
    pc[5] = -w[3] * s + w[4] * c;
}

/** focal distance of the action finder at a point with potential Phi: E, Lz -> Lcirc(E) ->
    (xi, chi) -> Delta; reference ActionFinderAxisymFudge::eval steps 0-1,
    src/actions_staeckel.cpp:957-977 */
static __device__ double finderFocalDistance(const FudgeTables& F, const double* pc, double Phi)
{
    const double E = Phi + 0.5 * (pc[3] * pc[3] + pc[4] * pc[4] + pc[5] * pc[5]);
    const double Lz = pc[0] * pc[5];
    const double Lcirc = interpLcirc(F, E);
    const double xi = clip(log(F.invPhi0 - 1 / E), ldg(F.gridE), ldg(F.gridE + F.nE - 1));
    const double Lzrel = clip(fabs(Lz) / Lcirc, 0., 1.);
    const double chi = scaleCub(0, 1, Lzrel);
    return fmax(0., deltaLookup(F, xi, chi));
}

}  // namespace agb
