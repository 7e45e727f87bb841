// Shared host/device numerics of the B200 engine: grid search, quintic/cubic Hermite
// segments, the hybrid Brent/Hermite root finder and the interval scalings.
//
// Each routine restates the algorithm of the reference library so that results agree with
// it to round-off; the reference location is given next to each one.
#pragma once
#include <cmath>
#include <cstdint>
#include <cfloat>

#ifdef __CUDACC__
#define AGB_HD __host__ __device__ __forceinline__
#else
#define AGB_HD inline
#endif

namespace agb {

/// largest spherical-harmonic order supported by the device tables
constexpr int LMAX_MAX = 16;
/// number of doubles stored per node of a 2-D quintic spline (9 used + 1 pad for 16-byte loads)
constexpr int NODE_STRIDE = 10;
/// most azimuthal harmonics the register-resident spline evaluator handles
constexpr int FAST_MAX_HARMONICS = 8;

/// sqrt(pi) to the digits the reference library uses (its M_SQRTPI)
constexpr double SQRT_PI = 1.77245385090551602729816748334;

AGB_HD double pow2(double x) { return x * x; }
AGB_HD double signOf(double x) { return x > 0 ? 1. : x < 0 ? -1. : 0.; }
AGB_HD bool isFinite(double x) { return x == x && x != INFINITY && x != -INFINITY; }
/// clamp to [lo, hi]; NaN maps to lo (as math::clip, reference src/math_core.h:29)
AGB_HD double clip(double x, double lo, double hi) { return x > hi ? hi : x > lo ? x : lo; }
AGB_HD bool signBit(double x) {
#ifdef __CUDA_ARCH__
    return signbit(x);
#else
    return std::signbit(x);
#endif
}

/** Index of the grid segment containing x: arr[i] <= x < arr[i+1]; -1 if x < arr[0] (or NaN),
    size-1 if x > arr[size-1]; x == arr[size-1] maps to the last segment (size-2).
    Starts from the guess of an equally-spaced grid, then bisects.
    Semantics of math::binSearch, reference src/math_core.cpp:251-280. */
AGB_HD int binSearch(double x, const double* arr, int size)
{
    if(size < 1 || !(x >= arr[0]))
        return -1;
    if(x > arr[size-1] || size < 2)
        return size - 1;
    int lo = static_cast<int>((x - arr[0]) / (arr[size-1] - arr[0]) * (size - 1));
    if(lo == size - 1)
        return size - 2;
    int hi = size - 1;
    if(x >= arr[lo]) {
        if(x < arr[lo+1])
            return lo;
    } else {
        hi = lo;
        lo = 0;
    }
    while(hi > lo + 1) {
        int mid = (hi + lo) / 2;
        if(arr[mid] > x) hi = mid; else lo = mid;
    }
    return lo;
}

/** binSearch with the first guess from scale = (size - 1) / (arr[size-1] - arr[0]), precomputed,
    instead of a division, and up to three steps to a neighbouring segment before the bisection
    (the grids are close to uniform: the guess is off by at most one or two segments); the guess
    and the steps only choose where the search looks, so the result is that of binSearch (the last
    segment whose left node is <= x). */
AGB_HD int binSearchScaled(double x, const double* arr, int size, double scale)
{
    if(size < 1 || !(x >= arr[0]))
        return -1;
    if(x > arr[size-1] || size < 2)
        return size - 1;
    int lo = static_cast<int>((x - arr[0]) * scale);
    if(lo >= size - 1)
        return size - 2;
    for(int step = 0; step < 3; step++) {
        if(x < arr[lo]) lo--;                               // lo > 0 here, since x >= arr[0]
        else if(lo < size - 2 && x >= arr[lo+1]) lo++;
        else return lo;
    }
    int hi = size - 1;
    if(x >= arr[lo]) {
        if(lo == size - 2 || x < arr[lo+1])
            return lo;
    } else {
        hi = lo;
        lo = 0;
    }
    while(hi > lo + 1) {
        int mid = (hi + lo) / 2;
        if(arr[mid] > x) hi = mid; else lo = mid;
    }
    return lo;
}

/** Quintic Hermite interpolation of K functions on the segment [xl, xh] from the values and the
    first and second derivatives at both ends; returns f, f', f'' (each output may be null).
    The polynomial is written as the Taylor part at xl plus corrections in the three
    "defects" (mismatch of f, f', f'' at xh), each multiplied by a fixed basis polynomial in t.
    Same interpolant and special case x == xh as evalQuinticSplines, reference
    src/math_spline.cpp:654-731. */
template<int K, typename T = double>
AGB_HD void quinticSegmentR(T x, T xl, T xh, T hi,
    const T* fl, const T* fh, const T* f1l, const T* f1h,
    const T* f2l, const T* f2h, T* f, T* df, T* d2f);

template<int K, typename T = double>
AGB_HD void quinticSegment(T x, T xl, T xh,
    const T* fl, const T* fh, const T* f1l, const T* f1h,
    const T* f2l, const T* f2h, T* f, T* df, T* d2f)
{
    quinticSegmentR<K, T>(x, xl, xh, 1 / (xh - xl), fl, fh, f1l, f1h, f2l, f2h, f, df, d2f);
}

/// the same with the reciprocal width hi = 1 / (xh - xl) given (tabulated per grid interval: the
/// correctly rounded reciprocal, so the results are those of quinticSegment bit for bit)
template<int K, typename T>
AGB_HD void quinticSegmentR(T x, T xl, T xh, T hi,
    const T* fl, const T* fh, const T* f1l, const T* f1h,
    const T* f2l, const T* f2h, T* f, T* df, T* d2f)
{
    if(x == xh) {   // exactly at the right node: return the node values without round-off
#pragma unroll
        for(int k = 0; k < K; k++) {
            if(f)   f[k]   = fh[k];
            if(df)  df[k]  = f1h[k];
            if(d2f) d2f[k] = f2h[k];
        }
        return;
    }
    const T dx = x - xl, hdx2 = T(0.5) * dx * dx, h = xh - xl, h2 = h * h;
    const T t = dx * hi, t2 = t * t, t3 = t * t2, omt = t * (1 - t);
    // basis polynomials for the three defects and their first two derivatives
    const T bf   = t3 * (10 - t * (15 - 6 * t));
    const T b1   = t3 * (1 - t * T(0.5)) * h;
    const T b2   = t3 * (1 - t * (T(1.25) - T(0.5) * t)) * h2;
    const T cx   = 30 * omt * hi;
    const T bfp  = cx * omt;
    const T b1p  = t2 * (3 - t * 2);
    const T b2p  = t2 * (3 - t * (5 - T(2.5) * t)) * h;
    const T bfpp = cx * hi * (2 - 4 * t);
    const T b1pp = cx * T(0.2);
    const T b2pp = t * (6 - t * (15 - 10 * t));
#pragma unroll
    for(int k = 0; k < K; k++) {
        const T d0 = fh[k]  - fl[k]  - T(0.5) * h * (f1h[k] + f1l[k]);
        const T d1 = f1h[k] - f1l[k] - T(0.5) * h * (f2h[k] + f2l[k]);
        const T d2 = f2h[k] - f2l[k];
        if(f)   f[k]   = fl[k] + bf * d0 + dx * f1l[k] + b1 * d1 + hdx2 * f2l[k] + b2 * d2;
        if(df)  df[k]  = bfp * d0 + f1l[k] + b1p * d1 + dx * f2l[k] + b2p * d2;
        if(d2f) d2f[k] = bfpp * d0 + b1pp * d1 + f2l[k] + b2pp * d2;
    }
}

/** Cubic Hermite interpolation of one function on [xl, xh] from values and first derivatives;
    same interpolant as evalCubicSplines, reference src/math_spline.cpp:593-651. */
AGB_HD void cubicSegment(double x, double xl, double xh, double fl, double fh, double dl, double dh,
    double* f, double* df, double* d2f)
{
    const double h = xh - xl, hi = 1 / h, t = (x - xl) / h, T = 1 - t, tT = t * T;
    const double dif = fh - fl, Q = 3 * (dl + dh) - 6 * hi * dif;
    if(f)   *f   = fl * T + fh * t + (dif * (t - T) + (dl * T - dh * t) * h) * tT;
    if(df)  *df  = dl * T + dh * t - Q * tT;
    if(d2f) *d2f = (dh - dl + Q * (t - T)) * hi;
}

// ------------------------------------------------------------------------------------------
// Interval scalings (reference src/math_core.cpp:296-396)

/// u in [u0, +inf): s = ln(u/u0) / (1 + ln(u/u0));  u0 > 0 (u0 == 0 uses the doubly-infinite map)
AGB_HD double unscaleSemiInf(double u0, double s, double* duds)
{
    if(u0 == 0) {
        double u = exp(1 / (1 - s) - 1 / s);
        if(signBit(u0)) u = -1 / u;
        if(duds) *duds = fabs(u) * (1 / pow2(1 - s) + 1 / pow2(s));
        return u;
    }
    double u = u0 * exp(s / (1 - s));
    if(duds) *duds = u / pow2(1 - s);
    return u;
}

/// u in (-inf, +inf): u = 1/(1-s) - 1/s
AGB_HD double unscaleInf(double s, double* duds)
{
    if(duds) *duds = 1 / pow2(1 - s) + 1 / pow2(s);
    return 1 / (1 - s) - 1 / s;
}

/// u in [ul, ur] with a cubic stretch near both ends: u = ul (1-s)^2 (1+2s) + ur s^2 (3-2s)
AGB_HD double unscaleCub(double ul, double ur, double s, double* duds)
{
    if(duds) *duds = (ur - ul) * 6 * s * (1 - s);
    return ul * pow2(1 - s) * (1 + 2 * s) + ur * pow2(s) * (3 - 2 * s);
}

/// inverse of unscaleCub: two Newton steps from an accurate initial guess
AGB_HD double scaleCub(double ul, double ur, double u)
{
    if(u == ul) return 0;
    if(u == ur) return 1;
    const double half = 0.5 * (ul + ur);
    if(u == half) return 0.5;
    const double w = u < half ? (u - ul) / (ur - ul) : (ur - u) / (ur - ul);
    double s = 0.5773502691896257 * sqrt(w) + w * (0.1184 + 0.1291 * w);
    for(int i = 0; i < 2; i++)
        s -= (1. / 6) * (s * s * (3 - 2 * s) - w) / (s * (1 - s));
    return u < half ? s : 1 - s;
}

// ------------------------------------------------------------------------------------------
// Root finder (reference src/math_core.cpp:866-1041: hybrid of Brent's method and a
// monotone Hermite-interpolation step when derivatives are available)

/// Hermite cubic through (x1,f1,d1), (x2,f2,d2) evaluated at x
AGB_HD double hermiteCubic(double x, double x1, double x2, double f1, double f2, double d1, double d2)
{
    const double h = x2 - x1, t = (x - x1) / h, T = 1 - t;
    return f1 * T * T * (1 + 2 * t) + f2 * t * t * (1 + 2 * T) + d1 * h * T * T * t - d2 * h * t * t * T;
}

/// the same, but NaN if the cubic is not monotone on [x1, x2]
AGB_HD double hermiteMonotone(double x, double x1, double x2, double f1, double f2, double d1, double d2)
{
    if(!isFinite(d1 + d2) || (d1 >= 0 && d2 < 0) || (d2 >= 0 && d1 < 0))
        return NAN;
    const double dx = x2 - x1;
    const double ai = 1 / (-6 * (f2 - f1) / dx + 3 * (d1 + d2));
    const double ba = -1 + (d2 - d1) * ai, ca = d1 * ai, D = pow2(ba) - 4 * ca;
    if(!isFinite(ba + D))
        return NAN;
    if(D >= 0) {
        const double sq = sqrt(D), t1 = 0.5 * (-ba - sq), t2 = 0.5 * (-ba + sq);
        if((t1 >= 0 && t1 <= 1) || (t2 >= 0 && t2 <= 1))
            return NAN;
    }
    return hermiteCubic(x, x1, x2, f1, f2, d1, d2);
}

constexpr int ROOT_MAXITER = 64;
constexpr double ROOT_DELTA_HERMITE = 1e-12;

/** Find a root of F on [xlower, xupper] to relative tolerance reltol (w.r.t. the interval width).
    F provides  void operator()(double x, double* f, double* dfdx) const  and the static
    constant  F::hasDeriv.  Returns NaN if the endpoints do not bracket a root or F is not finite.
    *numIter (if given) receives the number of iterations.  Algorithm of math::findRoot,
    reference src/math_core.cpp:895-1041 (MAXITER = 64, src/math_core.cpp:33). */
template<class F>
AGB_HD double findRoot(const F& fnc, double xlower, double xupper, double reltol, int* numIter = nullptr)
{
    const bool useDer = F::hasDeriv;
    double a = xlower, b = xupper, fa, fb, da = NAN, db = NAN;
    fnc(a, &fa, useDer ? &da : nullptr);
    fnc(b, &fb, useDer ? &db : nullptr);
    if(numIter) *numIter = 0;
    if((fa < 0 && fb < 0) || (fa > 0 && fb > 0) || !isFinite(fa + fb))
        return NAN;
    if(fa == 0)
        return fb == 0 ? 0.5 * (a + b) : a;
    if(fb == 0)
        return b;
    double c = a, fc = fa, dc = da, d = b - c, e = b - c;
    if(fabs(fc) < fabs(fb)) {
        a = b; b = c; c = a;  fa = fb; fb = fc; fc = fa;  da = db; db = dc; dc = da;
    }
    int iter = 0;
    const double abstol = fabs(xlower - xupper) * reltol;
    while(true) {
        const double tol = 0.5 * DBL_EPSILON * fabs(b), cb = c - b, m = 0.5 * cb;
        if(fb == 0 || fabs(m) <= tol)
            break;
        if(fabs(e) < tol || fabs(fa) <= fabs(fb)) {
            d = m; e = m;                                    // bisection
        } else {
            double dd = NAN;
            if(useDer && db * dc > 0)                        // inverse Hermite interpolation
                dd = hermiteMonotone(0, fb, fc, 0, cb, 1 / db, 1 / dc);
            if(isFinite(dd) && fmin(fabs(dd), fabs(cb - dd)) > fabs(cb) * ROOT_DELTA_HERMITE) {
                d = dd;
            } else {                                         // secant / inverse quadratic
                double p, q, r, s = fb / fa;
                if(a == c) {
                    p = 2 * m * s;
                    q = 1 - s;
                } else {
                    q = fa / fc;
                    r = fb / fc;
                    p = s * (2 * m * q * (q - r) - (b - a) * (r - 1));
                    q = (q - 1) * (r - 1) * (s - 1);
                }
                if(p > 0) q = -q; else p = -p;
                if(2 * p < fmin(3 * m * q - fabs(tol * q), fabs(e * q))) {
                    e = d; d = p / q;
                } else {
                    d = m; e = m;
                }
            }
        }
        a = b; fa = fb; da = db;
        b += fabs(d) > tol ? d : (m > 0 ? tol : -tol);
        fnc(b, &fb, useDer ? &db : nullptr);
        if(!isFinite(fb)) { b = NAN; break; }
        if((fb < 0 && fc < 0) || (fb > 0 && fc > 0)) {       // root lies between a and the new b
            c = a; fc = fa; dc = da; d = b - c; e = b - c;
        }
        if(fabs(fc) < fabs(fb)) {
            a = b; b = c; c = a;  fa = fb; fb = fc; fc = fa;  da = db; db = dc; dc = da;
        }
        iter++;
        if(fabs(b - c) <= abstol) {                          // bracket small enough: final secant
            const double off = fb * (b - c) / (fc - fb);
            if((off > 0 && off < c - b) || (off < 0 && off > c - b))
                b += off;
            break;
        } else if(useDer) {                                  // Newton step within the bracket
            const double off = -fb / db;
            const bool inside = (off > 0 && off < c - b) || (off < 0 && off > c - b);
            if(inside && fabs(off) < abstol) {
                b += off;
                break;
            }
        }
        if(iter >= ROOT_MAXITER)
            break;
    }
    if(numIter) *numIter = iter;
    return b;
}

/** findRoot (with derivatives) as a resumable state machine: the caller evaluates the function
    wherever the search asks, so that lanes of a warp that run different searches, at different
    iterations, meet at one evaluation site.  Arithmetic and results are those of findRoot above:

        double x = s.start(lo, hi, reltol);
        while(true) { f(x, &fx, &dx); if(s.feed(fx, dx, &x)) break; }
        root = s.result; iterations = s.iter;                                               */
struct RootSearch {
    double a, b, c, fa, fb, fc, da, db, dc, d, e, abstol;
    double result;
    int iter, phase;     // phase 0: wants f(xlower), 1: f(xupper), 2: f(next iterate),
                         // 3: f(xlower) with f(xupper) already known

    AGB_HD double start(double xlower, double xupper, double reltol)
    {
        return startAbs(xlower, xupper, fabs(xlower - xupper) * reltol);
    }

    /// the same search with its tolerance given directly (a bracket narrowed inside the original
    /// one keeps the original bracket's tolerance)
    AGB_HD double startAbs(double xlower, double xupper, double tol)
    {
        a = xlower; b = xupper;
        abstol = tol;
        iter = 0; phase = 0;
        return a;
    }

    /// the same search with f, f' at the upper end already known (so the first point to evaluate
    /// is the lower end, returned)
    AGB_HD double startKnownUpper(double xlower, double xupper, double tol, double fupper, double dupper)
    {
        startAbs(xlower, xupper, tol);
        fb = fupper; db = dupper;
        phase = 3;
        return a;
    }

    /// the same search with f, f' at both ends already known: true when it has finished at once
    /// (result set), otherwise *xnext is the first point to evaluate
    AGB_HD bool startKnownEnds(double xlower, double xupper, double tol, double flower, double dlower,
        double fupper, double dupper, double* xnext)
    {
        if(setupKnownEnds(xlower, xupper, tol, flower, dlower, fupper, dupper)) return true;
        return propose(xnext);
    }

    /// the same set-up without the first iterate: true when it has finished at once; otherwise
    /// propose() gives the first point to evaluate
    AGB_HD bool setupKnownEnds(double xlower, double xupper, double tol, double flower, double dlower,
        double fupper, double dupper)
    {
        startAbs(xlower, xupper, tol);
        fa = flower; da = dlower; fb = fupper; db = dupper;
        return setup();
    }

    /// take f and f' at the requested point; true when the search has finished (result set),
    /// otherwise *xnext is the next point to evaluate
    AGB_HD bool feed(double fx, double dx, double* xnext)
    {
        const int r = take(fx, dx, xnext);
        return r == 0 ? true : r == 2 ? false : propose(xnext);
    }

    /// feed without the proposal of the next iterate: 0 when the search has finished (result set),
    /// 1 when the next point is due from propose(), 2 when *xnext already holds it (an end of the
    /// bracket to evaluate); feed = take followed by propose when it returns 1
    AGB_HD int take(double fx, double dx, double* xnext)
    {
        if(phase == 0) {
            fa = fx; da = dx;
            phase = 1;
            *xnext = b;
            return 2;
        }
        if(phase == 1) {
            fb = fx; db = dx;
            return setup() ? 0 : 1;
        }
        if(phase == 3) {
            fa = fx; da = dx;
            return setup() ? 0 : 1;
        }
        fb = fx; db = dx;
        if(!isFinite(fb)) { result = NAN; return 0; }
        if((fb < 0 && fc < 0) || (fb > 0 && fc > 0)) {
            c = a; fc = fa; dc = da; d = b - c; e = b - c;
        }
        if(fabs(fc) < fabs(fb)) {
            a = b; b = c; c = a;  fa = fb; fb = fc; fc = fa;  da = db; db = dc; dc = da;
        }
        iter++;
        if(fabs(b - c) <= abstol) {
            const double off = fb * (b - c) / (fc - fb);
            if((off > 0 && off < c - b) || (off < 0 && off > c - b))
                b += off;
            result = b;
            return 0;
        }
        const double off = -fb / db;
        const bool inside = (off > 0 && off < c - b) || (off < 0 && off > c - b);
        if(inside && fabs(off) < abstol) { result = b + off; return 0; }
        if(iter >= ROOT_MAXITER) { result = b; return 0; }
        return 1;
    }

    /// replace the first iterate, just proposed after both end values were known (phase 2, the
    /// bracket between a and c), by the guess t when t lies strictly inside the bracket: true and
    /// *xnext = t; the step to t counts as the last step (d, e) for the next interpolation test
    AGB_HD bool seed(double t, double* xnext)
    {
        if(phase != 2 || iter != 0 || !((t - a) * (c - t) > 0)) return false;
        d = t - a; e = d;
        b = t;
        *xnext = t;
        return true;
    }

    /// both end values known: the bracket checks and the first iterate
    AGB_HD bool begin(double* xnext)
    {
        if(setup()) return true;
        return propose(xnext);
    }

    /// both end values known: the bracket checks and the initial state (true when finished)
    AGB_HD bool setup()
    {
        if((fa < 0 && fb < 0) || (fa > 0 && fb > 0) || !isFinite(fa + fb)) { result = NAN; return true; }
        if(fa == 0) { result = fb == 0 ? 0.5 * (a + b) : a; return true; }
        if(fb == 0) { result = b; return true; }
        c = a; fc = fa; dc = da; d = b - c; e = b - c;
        if(fabs(fc) < fabs(fb)) {
            a = b; b = c; c = a;  fa = fb; fb = fc; fc = fa;  da = db; db = dc; dc = da;
        }
        phase = 2;
        return false;
    }

    /// the head of one iteration: convergence test and the next iterate
    AGB_HD bool propose(double* xnext)
    {
        const double tol = 0.5 * DBL_EPSILON * fabs(b), cb = c - b, m = 0.5 * cb;
        if(fb == 0 || fabs(m) <= tol) { result = b; return true; }
        if(fabs(e) < tol || fabs(fa) <= fabs(fb)) {
            d = m; e = m;
        } else {
            double dd = NAN;
            if(db * dc > 0)
                dd = hermiteMonotone(0, fb, fc, 0, cb, 1 / db, 1 / dc);
            if(isFinite(dd) && fmin(fabs(dd), fabs(cb - dd)) > fabs(cb) * ROOT_DELTA_HERMITE) {
                d = dd;
            } else {
                double p, q, r, s = fb / fa;
                if(a == c) {
                    p = 2 * m * s;
                    q = 1 - s;
                } else {
                    q = fa / fc;
                    r = fb / fc;
                    p = s * (2 * m * q * (q - r) - (b - a) * (r - 1));
                    q = (q - 1) * (r - 1) * (s - 1);
                }
                if(p > 0) q = -q; else p = -p;
                if(2 * p < fmin(3 * m * q - fabs(tol * q), fabs(e * q))) {
                    e = d; d = p / q;
                } else {
                    d = m; e = m;
                }
            }
        }
        a = b; fa = fb; da = db;
        b += fabs(d) > tol ? d : (m > 0 ? tol : -tol);
        *xnext = b;
        return false;
    }
};

}  // namespace agb
