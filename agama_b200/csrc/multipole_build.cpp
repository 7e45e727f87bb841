// Host-side construction of the Multipole tables from (radii, Phi_lm, dPhi_lm), and the
// coefficient-file reader.  Runs once per potential; the evaluation itself is device code.
#include "multipole.h"
#include "sphharm.cuh"
#include "ref_tables.h"
#include <stdexcept>
#include <fstream>
#include <sstream>
#include <algorithm>
#include <cstring>
#include <cstdio>
#include <cmath>

namespace agb {

namespace {

const double SQRT_DBL_EPSILON = 1.4901161193847656e-08;
const double ROOT3_DBL_EPSILON = 6.0554544523933395e-06;   // DBL_EPSILON^(1/3)
const double GRID_SAFETY_FACTOR = ROOT3_DBL_EPSILON;        // reference src/potential_multipole.cpp:59
const int LMAX_1D_SPLINE = 2;                               // reference src/potential_multipole.cpp:43


inline bool isXRefl(int s) { return (s & SYM_XREFL) == SYM_XREFL; }
inline bool isYRefl(int s) { return (s & SYM_YREFL) == SYM_YREFL; }
inline bool isZRefl(int s) { return (s & SYM_ZREFL) == SYM_ZREFL; }
inline bool isRefl (int s) { return (s & SYM_REFL)  == SYM_REFL; }
inline bool isBisym(int s) { return (s & (SYM_ZREFL | SYM_REFL)) == (SYM_ZREFL | SYM_REFL); }

/// Thomas algorithm for a tridiagonal system: sub-diagonal a, diagonal b, super-diagonal c
std::vector<double> solveTridiagonal(const std::vector<double>& a, const std::vector<double>& b,
    const std::vector<double>& c, const std::vector<double>& rhs)
{
    const size_t n = b.size();
    std::vector<double> cp(n), x(n);
    for(size_t i = 0; i < n; i++) {
        const double piv = 1. / (b[i] - (i > 0 ? a[i] * cp[i-1] : 0));
        cp[i] = c[i] * piv;
        x[i] = (rhs[i] - (i > 0 ? a[i] * x[i-1] : 0)) * piv;
    }
    for(size_t i = n - 1; i-- > 0; )
        x[i] -= cp[i] * x[i+1];
    return x;
}

/// brackets of the inner-monopole asymptote: the density ~ r^(s-2) + const condition
struct AsymptoteEquation {
    static constexpr bool hasDeriv = false;
    double coef, ratio, dPhi1, dPhi2;
    void operator()(double s, double* f, double*) const {
        const double rsm1 = pow(ratio, s - 1);
        *f = coef * (rsm1 - ratio) + (dPhi2 - dPhi1 * rsm1) * 0.5 * (pow2(ratio) - 1) +
             (dPhi1 * ratio - dPhi2) * (ratio * rsm1 - 1) / s;
    }
};

/** Power-law extrapolation coefficients of one harmonic from its values at two radii and the
    derivative at the first:  Phi = W (r/r1)^v + U (r/r1)^s [+ Q (r/r1)^2 for the inner monopole]
    (or U (r/r1)^s ln(r/r1) when s == v).  Reference computeExtrapolationCoefs,
    src/potential_multipole.cpp:553-614. */
void extrapolationCoefs(double Phi1, double Phi2, double dPhi1, double dPhi2, double r1, double r2,
    int v, double s0, double& s, double& U, double& W, double& Q)
{
    if(v == 0) {
        AsymptoteEquation eq{ (Phi2 - Phi1) / r1, r2 / r1, dPhi1, dPhi2 };
        s = findRoot(eq, 2 + 3 * SQRT_DBL_EPSILON, 8.0, SQRT_DBL_EPSILON);
        const double rsm1 = pow(r2 / r1, s - 1);
        U = (dPhi2 * r1 - dPhi1 * r2) / (rsm1 - r2 / r1) / s;
        Q = (dPhi1 * rsm1 - dPhi2) * r1 / (rsm1 - r2 / r1) * 0.5;
        const double rho0 = 6 * Q, rho1 = 6 * Q + s * (s + 1) * U;
        if(s == s && rho0 * rho1 > 0) {
            W = Phi1 - U - Q;
            return;
        }
        Q = 0;
    }
    const double lnr = log(r2 / r1);
    const double num1 = r1 * dPhi1, num2 = v * Phi1, den1 = Phi1, den2 = Phi2 * exp(-v * lnr);
    const double A = lnr * (num1 - num2) / (den1 - den2);
    const double SAFETY = 100 * DBL_EPSILON;
    const bool roundoff =
        fabs(num1 - num2) < std::max(fabs(num1), fabs(num2)) * SAFETY ||
        fabs(den1 - den2) < std::max(fabs(den1), fabs(den2)) * SAFETY;
    if(!isFinite(A) || A >= 0 || roundoff) {
        U = 0; s = 0; W = Phi1;
        return;
    }
    s = fabs(A + 1) < SQRT_DBL_EPSILON ? v : v + (A - lambertW(A * exp(A), A > -1)) / lnr;
    if(v >= 0 && !isFinite(s)) s = 2;
    if(v < 0 && (!isFinite(s) || s >= 0)) s = -2;
    if(v > 0)  s = fmax(s, s0);
    if(v < -1) s = fmin(s, s0);
    if(s != v) {
        U = (r1 * dPhi1 - v * Phi1) / (s - v);
        W = (r1 * dPhi1 - s * Phi1) / (v - s);
    } else {
        U = r1 * dPhi1 - v * Phi1;
        W = Phi1;
    }
}

MultipoleHost::Asympt makeAsymptote(const std::vector<double>& radii,
    const std::vector<std::vector<double>>& Phi, const std::vector<std::vector<double>>& dPhi, bool inner)
{
    const size_t nc = Phi.size();
    MultipoleHost::Asympt a;
    a.S.assign(nc, 0); a.U.assign(nc, 0); a.W.assign(nc, 0);
    const size_t i1 = inner ? 0 : Phi[0].size() - 1, i2 = inner ? 1 : Phi[0].size() - 2;
    double Q = 0;
    for(size_t c = 0; c < nc; c++) {
        const int l = static_cast<int>(sqrt(static_cast<double>(c)));
        extrapolationCoefs(Phi[c][i1], Phi[c][i2], dPhi[c][i1], dPhi[c][i2], radii[i1], radii[i2],
            inner ? l : -l - 1, a.S[0], a.S[c], a.U[c], a.W[c], Q);
    }
    a.Q = Q;
    a.inner = inner ? 1 : 0;
    a.r0sq = radii[i1] * radii[i1];
    a.ind = indicesFromCoefs(a.U);   // the expansion's term set follows the non-zero amplitudes U
    return a;
}

/** tau grid: Gauss-Legendre nodes in cos(theta) for lmax+1 points mapped to tau, plus the
    endpoints -1, 1, each interval split into 3; reference createGridInTau,
    src/potential_multipole.cpp:1828-1852 */
std::vector<double> gridInTau(int lmax)
{
    const int ngl = lmax + 1;
    if(ngl > GL_HALF_MAXN)
        throw std::invalid_argument("Multipole: lmax too large for the angular grid");
    std::vector<double> t(ngl + 2);
    const double* half = GL_HALF_NODES + GL_HALF_OFFSET[ngl];
    for(int i = 0; i <= ngl / 2; i++) {         // nodes on [-1, 1] from the rule on [0, 1]
        t[1 + i] = -1 + half[i] * 2;
        t[ngl - i] = 1 - half[i] * 2;
    }
    for(int i = 1; i <= ngl; i++)
        t[i] /= 1 + sqrt(1 - pow2(t[i]));
    t.front() = -1;
    t.back() = 1;
    const int over = 3, n = (ngl + 1) * over + 1;
    std::vector<double> g(n);
    for(int i = 0; i <= ngl; i++)
        for(int k = 0; k < over; k++)
            g[i * over + k] = (t[i] * (over - k) + t[i+1] * k) / over;
    g.back() = 1;
    return g;
}

void checkFiniteVec(const std::vector<double>& v, const char* what) {
    for(double x : v)
        if(!isFinite(x))
            throw std::invalid_argument(std::string("Multipole: non-finite values in ") + what);
}

/** 2-D quintic spline with given f, f_x, f_y, f_xy at nodes: the remaining derivatives come from
    1-D quintic splines along rows and columns; reference QuinticSpline2d::setupWithMixedDeriv,
    src/math_spline.cpp:2478-2533.  Input/output arrays are [nx][ny]. */
void setupQuintic2d(const std::vector<double>& xv, const std::vector<double>& yv,
    const std::vector<double>& f, const std::vector<double>& fx, const std::vector<double>& fy,
    const std::vector<double>& fxy, double* out /*[nx][ny][NODE_STRIDE]*/)
{
    const size_t nx = xv.size(), ny = yv.size(), n = nx * ny;
    std::vector<double> fxx(n), fyy(n), fxxy(n), fxyy(n), fxxyy(n);
    std::vector<double> t(nx), tx(nx), ty(nx), txy(nx);
    for(size_t j = 0; j < ny; j++) {
        for(size_t i = 0; i < nx; i++) {
            t[i] = f[i*ny+j]; tx[i] = fx[i*ny+j]; ty[i] = fy[i*ny+j]; txy[i] = fxy[i*ny+j];
        }
        std::vector<double> a = quinticSecondDerivs(xv, t, tx), b = quinticSecondDerivs(xv, ty, txy);
        for(size_t i = 0; i < nx; i++) { fxx[i*ny+j] = a[i]; fxxy[i*ny+j] = b[i]; }
    }
    std::vector<double> u(ny), ux(ny), uy(ny), uxx(ny), uxy(ny), uxxy(ny);
    for(size_t i = 0; i < nx; i++) {
        for(size_t j = 0; j < ny; j++) {
            u[j] = f[i*ny+j]; ux[j] = fx[i*ny+j]; uy[j] = fy[i*ny+j];
            uxx[j] = fxx[i*ny+j]; uxy[j] = fxy[i*ny+j]; uxxy[j] = fxxy[i*ny+j];
        }
        std::vector<double> a = quinticSecondDerivs(yv, u, uy), b = quinticSecondDerivs(yv, ux, uxy),
            c = quinticSecondDerivs(yv, uxx, uxxy);
        for(size_t j = 0; j < ny; j++) { fyy[i*ny+j] = a[j]; fxyy[i*ny+j] = b[j]; fxxyy[i*ny+j] = c[j]; }
    }
    for(size_t k = 0; k < n; k++) {
        double* o = out + k * NODE_STRIDE;
        o[0] = f[k]; o[1] = fx[k]; o[2] = fy[k]; o[3] = fxx[k]; o[4] = fxy[k];
        o[5] = fyy[k]; o[6] = fxxy[k]; o[7] = fxyy[k]; o[8] = fxxyy[k]; o[9] = 0;
    }
}

}  // namespace

// ------------------------------------------------------------------------------------------

double lambertW(double x, bool lowerBranch)
{
    // Halley iteration on w e^w = x; initial guesses from the branch-point series and the
    // asymptotic expansions (Corless et al. 1996)
    const double branchPoint = -0.36787944117144233;
    double w;
    if(!lowerBranch) {
        if(x < branchPoint) return NAN;
        if(x == 0) return 0;
        if(x == branchPoint) return -1;
        if(x < -0.25) {
            const double p = sqrt(2 * (2.718281828459045 * x + 1));
            w = -1 + p - p * p / 3 + 11. / 72 * p * p * p;
        } else if(x < 3) w = log1p(x) * (1 - log1p(log1p(x)) / (2 + log1p(x)));
        else { const double l1 = log(x), l2 = log(l1); w = l1 - l2 + l2 / l1; }
    } else {
        if(x < branchPoint || x >= 0) return x == 0 ? -INFINITY : NAN;
        if(x == branchPoint) return -1;
        if(x < -0.25) {
            const double p = -sqrt(2 * (2.718281828459045 * x + 1));
            w = -1 + p - p * p / 3 + 11. / 72 * p * p * p;
        } else { const double l1 = log(-x), l2 = log(-l1); w = l1 - l2 + l2 / l1; }
    }
    for(int i = 0; i < 100; i++) {
        const double ew = exp(w), f = w * ew - x, wp1 = w + 1;
        const double dw = f / (ew * wp1 - (w + 2) * f / (2 * wp1));
        w -= dw;
        if(fabs(dw) <= 4e-16 * (1 + fabs(w))) break;
    }
    return w;
}

void glNodesWeights(int n, double* nodes, double* weights)
{
    // Newton iteration on P_n(x) from the Chebyshev-like initial guesses; nodes ascending
    for(int i = 0; i < (n + 1) / 2; i++) {
        double x = cos(M_PI * (i + 0.75) / (n + 0.5)), dp = 0;
        for(int it = 0; it < 100; it++) {
            double p0 = 1, p1 = x;
            for(int k = 2; k <= n; k++) { const double p2 = ((2 * k - 1) * x * p1 - (k - 1) * p0) / k; p0 = p1; p1 = p2; }
            if(n == 1) { p1 = x; p0 = 1; }
            dp = n * (x * p1 - p0) / (x * x - 1);
            const double dx = p1 / dp;
            x -= dx;
            if(fabs(dx) < 1e-16) break;
        }
        double p0 = 1, p1 = x;
        for(int k = 2; k <= n; k++) { const double p2 = ((2 * k - 1) * x * p1 - (k - 1) * p0) / k; p0 = p1; p1 = p2; }
        dp = n * (x * p1 - p0) / (x * x - 1);
        const double w = 2 / ((1 - x * x) * dp * dp);
        nodes[i] = -x; nodes[n - 1 - i] = x;
        weights[i] = weights[n - 1 - i] = w;
    }
    if(n % 2 == 1) nodes[n / 2] = 0;
}

/** Second derivatives of a quintic spline through (x, f) with given first derivatives, from
    continuity of f''' at interior nodes and f'''' = 0 at both ends (tridiagonal system);
    reference constructQuinticSpline(x, f, f'), src/math_spline.cpp:455-486. */
std::vector<double> quinticSecondDerivs(const std::vector<double>& x, const std::vector<double>& f,
    const std::vector<double>& d)
{
    const size_t n = x.size();
    if(n < 2) return std::vector<double>(n, 0);
    std::vector<double> lo(n, 0), di(n, 0), up(n, 0), rhs(n, 0);
    for(size_t i = 0; i < n; i++) {
        if(i > 0) {
            const double hi = 1 / (x[i] - x[i-1]);
            di[i] += hi * 3;
            rhs[i] -= (20 * (f[i] - f[i-1]) * hi - 12 * d[i] - 8 * d[i-1]) * hi * hi;
        }
        if(i < n - 1) {
            const double hi = 1 / (x[i+1] - x[i]);
            di[i] += hi * 3;
            up[i] = -hi;
            lo[i+1] = -hi;
            rhs[i] += (20 * (f[i+1] - f[i]) * hi - 12 * d[i] - 8 * d[i+1]) * hi * hi;
        }
    }
    double hi = 1 / (x[1] - x[0]);
    up[0] = -2 * hi;
    rhs[0] = (30 * (f[1] - f[0]) * hi - 14 * d[1] - 16 * d[0]) * hi * hi;
    hi = 1 / (x[n-1] - x[n-2]);
    lo[n-1] = -2 * hi;
    rhs[n-1] = (-30 * (f[n-1] - f[n-2]) * hi + 14 * d[n-2] + 16 * d[n-1]) * hi * hi;
    return solveTridiagonal(lo, di, up, rhs);
}

HarmIndices makeIndices(int lmax, int mmax, int sym)
{
    if(lmax < 0 || mmax < 0 || mmax > lmax || lmax > LMAX_MAX)
        throw std::invalid_argument("Multipole: unsupported order of expansion");
    HarmIndices h;
    h.lmax = lmax; h.mmax = mmax;
    h.step = (isZRefl(sym) || isRefl(sym)) ? 2 : 1;
    if(mmax == 0) sym |= SYM_ZROT | SYM_XREFL | SYM_YREFL;
    if(lmax == 0) sym |= SYM_ROT | SYM_ZREFL | SYM_REFL;
    h.sym = sym;
    for(int m = -mmax; m <= mmax; m++) {
        int lm = std::abs(m);
        if(isRefl(sym) && m % 2 != 0) lm = std::abs(m) + 1;
        if((isYRefl(sym) && m < 0) || (isXRefl(sym) && ((m < 0) ^ (m % 2 != 0))) || (isBisym(sym) && m % 2 != 0))
            lm = lmax + 1;
        h.lminArr[m + mmax] = lm;
    }
    return h;
}

/// symmetry and order of an expansion from the pattern of its non-zero coefficients;
/// reference getIndicesFromCoefs, src/math_sphharm.cpp:206-230
HarmIndices indicesFromCoefs(const std::vector<double>& C)
{
    const int lmax = static_cast<int>(sqrt(static_cast<double>(C.size()))) - 1;
    if(lmax < 0 || static_cast<int>(C.size()) != (lmax + 1) * (lmax + 1))
        throw std::invalid_argument("Multipole: invalid size of coefficient array");
    int sym = SYM_SPHERICAL, mmax = 0;
    for(size_t c = 0; c < C.size(); c++) {
        if(!isFinite(C[c]))
            throw std::domain_error("Multipole: coefficient not finite");
        if(C[c] != 0) {
            const int l = static_cast<int>(sqrt(static_cast<double>(c))), m = static_cast<int>(c) - l * (l + 1);
            if(l % 2 == 1) sym &= ~SYM_REFL;
            if(m < 0) sym &= ~SYM_YREFL;
            if((l + m) % 2 == 1) sym &= ~SYM_ZREFL;
            if((m < 0) ^ (m % 2 != 0)) sym &= ~SYM_XREFL;
            if(m != 0) { sym &= ~SYM_ZROT; mmax = std::max(mmax, std::abs(m)); }
            if(l > 0) sym &= ~SYM_ROT;
        }
    }
    return makeIndices(lmax, mmax, sym);
}

MultipoleHost buildMultipole(const std::vector<double>& radii,
    const std::vector<std::vector<double>>& Phi, const std::vector<std::vector<double>>& dPhi)
{
    MultipoleHost M;
    const size_t nr = radii.size(), nc = Phi.size();
    bool ok = nr >= 2 && nc >= 1 && dPhi.size() == nc;
    for(size_t c = 0; ok && c < nc; c++)
        ok = Phi[c].size() == nr && dPhi[c].size() == nr;
    for(size_t k = 1; ok && k < nr; k++)
        ok = radii[k] > radii[k-1];
    if(!ok || !(radii[0] > 0))
        throw std::invalid_argument("Multipole: invalid radial grid");
    std::vector<double> D(nc, 0);
    for(size_t c = 0; c < nc; c++)
        for(size_t k = 0; k < nr; k++)
            D[c] += fabs(Phi[c][k]) + fabs(dPhi[c][k]);
    M.ind = indicesFromCoefs(D);
    const HarmIndices& ind = M.ind;
    M.radii = radii;
    M.Phi = Phi;
    M.dPhi = dPhi;
    M.lnr.resize(nr);
    for(size_t k = 0; k < nr; k++) M.lnr[k] = log(radii[k]);
    for(int i = 0; i < 2 * LMAX_MAX + 1; i++) M.splSlot[i] = -1;

    // inner value of the monopole (for the log-scaling of the amplitude)
    double s, U, W, Q;
    extrapolationCoefs(Phi[0][0], Phi[0][1], dPhi[0][0], dPhi[0][1], radii[0], radii[1], 0, NAN, s, U, W, Q);
    M.invPhi0 = s > 0 ? 1. / W : 0;
    M.logScaling = 1;

    if(ind.lmax <= LMAX_1D_SPLINE) {
        // ---- 1-D quintic splines in ln r per (l,m); reference MultipoleInterp1d ctor :1691-1747
        M.is2d = 0;
        for(size_t k = 0; k < nr; k++) {
            M.logScaling &= Phi[0][k] < 0;
            if(Phi[0][k] * M.invPhi0 >= 1) M.invPhi0 = 0;
        }
        M.spl1d.assign(nc * nr * 3, 0);
        std::vector<double> f(nr), d(nr);
        for(int m = ind.mmin(); m <= ind.mmax; m++)
            for(int l = ind.lmin(m); l <= ind.lmax; l += ind.step) {
                const int c = HarmIndices::index(l, m);
                for(size_t k = 0; k < nr; k++) {
                    if(M.logScaling) {
                        if(c == 0) {
                            f[k] = log(M.invPhi0 - 1 / Phi[c][k]);
                            d[k] = radii[k] * dPhi[c][k] / (Phi[c][k] * (M.invPhi0 * Phi[c][k] - 1));
                        } else {
                            f[k] = Phi[c][k] / Phi[0][k];
                            d[k] = (dPhi[c][k] - f[k] * dPhi[0][k]) * radii[k] / Phi[0][k];
                        }
                    } else {
                        f[k] = Phi[c][k];
                        d[k] = radii[k] * dPhi[c][k];
                    }
                }
                checkFiniteVec(f, "fvalues");
                checkFiniteVec(d, "fderivs");
                std::vector<double> d2 = quinticSecondDerivs(M.lnr, f, d);
                for(size_t k = 0; k < nr; k++) {
                    M.spl1d[(c * nr + k) * 3 + 0] = f[k];
                    M.spl1d[(c * nr + k) * 3 + 1] = d[k];
                    M.spl1d[(c * nr + k) * 3 + 2] = d2[k];
                }
            }
    } else {
        // ---- 2-D quintic splines in (ln r, tau) per m; reference MultipoleInterp2d ctor :1854-1967
        M.is2d = 1;
        M.tau = gridInTau(ind.lmax);
        const size_t nt = M.tau.size(), n = nr * nt;
        std::vector<double> val(n), dR(n), dT(n), dRdT(n), v0, dR0, dT0, dRdT0;
        std::vector<double> P(ind.lmax + 1), dP(ind.lmax + 1);
        std::vector<std::vector<double>> slots;
        for(int mm = 0; mm <= ind.mmax - ind.mmin(); mm++) {
            const int m = mm <= ind.mmax ? mm : ind.mmax - mm;   // m = 0 first
            const int lmin = ind.lmin(m);
            if(lmin > ind.lmax) continue;
            const int absm = std::abs(m);
            const double mul = m == 0 ? 2 * SQRT_PI : 2 * SQRT_PI * M_SQRT2;
            for(size_t j = 0; j < nt; j++) {
                legendreArray(ind.lmax, absm, M.tau[j], &P[0], &dP[0], nullptr);
                for(size_t k = 0; k < nr; k++) {
                    double v = 0, r = 0, t = 0, rt = 0;
                    for(int l = lmin; l <= ind.lmax; l += ind.step) {
                        const int c = HarmIndices::index(l, m);
                        v  +=  Phi[c][k] *  P[l - absm];
                        r  += dPhi[c][k] *  P[l - absm];
                        t  +=  Phi[c][k] * dP[l - absm];
                        rt += dPhi[c][k] * dP[l - absm];
                    }
                    if(m == 0) {
                        M.logScaling &= v < 0;
                        if(M.invPhi0 <= 1 / (mul * v)) M.invPhi0 = 0;
                    }
                    const size_t i = k * nt + j;
                    val[i]  = mul * v;
                    dR[i]   = mul * r * radii[k];
                    dT[i]   = mul * t * -2 / (pow2(M.tau[j]) + 1);
                    dRdT[i] = mul * rt * radii[k] * -2 / (pow2(M.tau[j]) + 1);
                }
            }
            if(m == 0) {
                v0 = val; dR0 = dR; dT0 = dT; dRdT0 = dRdT;
                if(M.logScaling) {
                    for(size_t i = 0; i < n; i++) {
                        const double q = 1 / (v0[i] * (M.invPhi0 * v0[i] - 1));
                        dR[i] *= q;
                        dT[i] *= q;
                        dRdT[i] = q * dRdT[i] + (1 - 2 * M.invPhi0 * v0[i]) * dR[i] * dT[i];
                        val[i] = log(M.invPhi0 - 1 / v0[i]);
                    }
                }
            } else if(M.logScaling) {
                for(size_t i = 0; i < n; i++) {
                    const double rel = val[i] / v0[i];
                    val[i] = rel;
                    dR[i] = (dR[i] - rel * dR0[i]) / v0[i];
                    dT[i] = (dT[i] - rel * dT0[i]) / v0[i];
                    dRdT[i] = (dRdT[i] - rel * dRdT0[i] - dR[i] * dT0[i] - dT[i] * dR0[i]) / v0[i];
                }
            }
            checkFiniteVec(val, "fvalues"); checkFiniteVec(dR, "dfdx");
            checkFiniteVec(dT, "dfdy");     checkFiniteVec(dRdT, "d2fdxdy");
            std::vector<double> tab(n * NODE_STRIDE);
            setupQuintic2d(M.lnr, M.tau, val, dR, dT, dRdT, &tab[0]);
            M.splSlot[m + ind.mmax] = static_cast<int>(slots.size());
            slots.push_back(tab);
        }
        M.numSlots = static_cast<int>(slots.size());
        for(auto& t : slots) M.spl2d.insert(M.spl2d.end(), t.begin(), t.end());
    }
    M.inner = makeAsymptote(radii, Phi, dPhi, true);
    M.outer = makeAsymptote(radii, Phi, dPhi, false);
    // sanity check of the asymptotic slopes (reference PowerLawMultipole ctor :1589-1597)
    (void)GRID_SAFETY_FACTOR;
    return M;
}

// ------------------------------------------------------------------------------------------
// coefficient file

namespace {
std::vector<std::string> splitTabs(const std::string& line) {
    std::vector<std::string> out;
    std::string cur;
    for(char ch : line) {
        if(ch == '\t' || ch == ' ') { if(!cur.empty()) { out.push_back(cur); cur.clear(); } }
        else cur += ch;
    }
    if(!cur.empty()) out.push_back(cur);
    return out;
}
std::string trim(const std::string& s) {
    size_t a = s.find_first_not_of(" \t\r"), b = s.find_last_not_of(" \t\r");
    return a == std::string::npos ? "" : s.substr(a, b - a + 1);
}
std::string lower(std::string s) { for(auto& c : s) c = static_cast<char>(tolower(c)); return s; }

/// parse a block "#radius\tl=0,m=0\t..." followed by gridSize rows
void parseBlock(const std::vector<std::string>& lines, size_t& pos, size_t gridSize,
    std::vector<double>& radii, std::vector<std::vector<double>>& coefs)
{
    if(pos >= lines.size() || lines[pos].empty() || lines[pos][0] != '#')
        throw std::runtime_error("Multipole coefficient file: missing header line");
    std::vector<std::string> head = splitTabs(lines[pos++]);
    // header columns l=..,m=..  define the coefficient index l*(l+1)+m
    std::vector<int> idx;
    for(size_t i = 1; i < head.size(); i++) {
        int l = 0, m = 0;
        if(sscanf(head[i].c_str(), "l=%d,m=%d", &l, &m) != 2)
            throw std::runtime_error("Multipole coefficient file: bad column header " + head[i]);
        idx.push_back(l * (l + 1) + m);
    }
    int ncoef = 0;
    for(int c : idx) ncoef = std::max(ncoef, c + 1);
    const int lmax = static_cast<int>(ceil(sqrt(static_cast<double>(ncoef)))) - 1;
    coefs.assign((lmax + 1) * (lmax + 1), std::vector<double>(gridSize, 0));
    radii.assign(gridSize, 0);
    for(size_t k = 0; k < gridSize; k++) {
        if(pos >= lines.size())
            throw std::runtime_error("Multipole coefficient file: too few rows");
        std::vector<std::string> f = splitTabs(lines[pos++]);
        if(f.size() != idx.size() + 1)
            throw std::runtime_error("Multipole coefficient file: wrong number of columns");
        radii[k] = strtod(f[0].c_str(), nullptr);
        for(size_t i = 0; i < idx.size(); i++)
            coefs[idx[i]][k] = strtod(f[i + 1].c_str(), nullptr);
    }
}
}  // namespace

namespace {
/// names of the symmetry types as the reference writes them (getSymmetryNameByType,
/// src/potential_factory.cpp:240-252); other combinations as their number
std::string symmetryName(int sym)
{
    switch(sym) {
        case SYM_NONE: return "None";
        case SYM_REFL: return "Reflection";
        case SYM_XREFL | SYM_YREFL | SYM_REFL: return "Bisymmetric";
        case SYM_TRIAXIAL: return "Triaxial";
        case SYM_AXISYMMETRIC: return "Axisymmetric";
        case SYM_SPHERICAL: return "Spherical";
        default: return std::to_string(sym);
    }
}

void writeBlock(std::ostream& out, const std::vector<double>& radii, const std::vector<std::vector<double>>& coefs)
{
    const int lmax = static_cast<int>(std::lround(std::sqrt(static_cast<double>(coefs.size())))) - 1;
    out << "#radius";
    for(int l = 0; l <= lmax; l++)
        for(int m = -l; m <= l; m++) out << "\tl=" << l << ",m=" << m;
    out << '\n';
    char buf[40];
    for(size_t k = 0; k < radii.size(); k++) {
        snprintf(buf, sizeof(buf), "%.17g", radii[k]);
        out << buf;
        for(size_t c = 0; c < coefs.size(); c++) {
            const double v = k < coefs[c].size() ? coefs[c][k] : 0;
            if(v == 0) out << "\t0";
            else { snprintf(buf, sizeof(buf), "%.17g", v); out << '\t' << buf; }
        }
        out << '\n';
    }
}
}  // namespace

void writeMultipoleCoefFile(const std::string& fileName, const std::vector<double>& radii,
    const std::vector<std::vector<double>>& Phi, const std::vector<std::vector<double>>& dPhi, int symmetry)
{
    if(radii.size() < 2 || Phi.empty() || Phi.size() != dPhi.size())
        throw std::invalid_argument("writeMultipoleCoefFile: inconsistent coefficients");
    const size_t nc = Phi.size();
    const size_t lp1 = static_cast<size_t>(std::lround(std::sqrt(static_cast<double>(nc))));
    if(lp1 * lp1 != nc)
        throw std::invalid_argument("writeMultipoleCoefFile: the number of coefficients is not (lmax+1)^2");
    std::ofstream out(fileName);
    if(!out)
        throw std::runtime_error("cannot write " + fileName);
    out << "[Potential]\ntype=Multipole\ngridSizeR=" << radii.size() << "\nlmax=" << (lp1 - 1) << "\nsymmetry="
        << symmetryName(symmetry) << "\nCoefficients\n#Phi\n";
    writeBlock(out, radii, Phi);
    out << "\n#dPhi/dr\n";
    writeBlock(out, radii, dPhi);
    if(!out)
        throw std::runtime_error("error writing " + fileName);
}

void readMultipoleCoefFile(const std::string& fileName, std::vector<double>& radii,
    std::vector<std::vector<double>>& Phi, std::vector<std::vector<double>>& dPhi)
{
    std::ifstream in(fileName);
    if(!in)
        throw std::runtime_error("cannot open " + fileName);
    std::vector<std::string> lines;
    std::string line;
    while(std::getline(in, line)) lines.push_back(trim(line));
    size_t gridSize = 0, pos = 0;
    bool isMultipole = false;
    for(; pos < lines.size(); pos++) {
        const std::string l = lower(lines[pos]);
        if(l.rfind("type=", 0) == 0) isMultipole = l.substr(5) == "multipole";
        if(l.rfind("gridsizer=", 0) == 0) gridSize = static_cast<size_t>(atol(l.substr(10).c_str()));
        if(l == "coefficients") { pos++; break; }
    }
    if(!isMultipole || gridSize < 2)
        throw std::runtime_error("not a Multipole coefficient file: " + fileName);
    while(pos < lines.size() && lines[pos] != "#Phi") pos++;
    if(pos >= lines.size()) throw std::runtime_error("Multipole coefficient file: no #Phi block");
    pos++;
    parseBlock(lines, pos, gridSize, radii, Phi);
    while(pos < lines.size() && lines[pos] != "#dPhi/dr") pos++;
    if(pos >= lines.size()) throw std::runtime_error("Multipole coefficient file: no #dPhi/dr block");
    pos++;
    std::vector<double> r2;
    parseBlock(lines, pos, gridSize, r2, dPhi);
    if(dPhi.size() != Phi.size())
        throw std::runtime_error("Multipole coefficient file: inconsistent blocks");
}

}  // namespace agb
