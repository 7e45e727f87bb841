// Project-written implementation of the small part of the GSL API that the reference
// Agama sources reach while constructing the benchmark potentials and action finders.
//
// TEST INFRASTRUCTURE ONLY (oracle build): nothing in the B200 engine links this file.
// Implemented from the mathematics, not from GSL sources:
//   * Lambert W (branches 0 and -1): Halley iteration on w e^w = x (Corless et al. 1996).
//   * Gamma family: std::tgamma / std::lgamma; the regularised upper incomplete gamma by
//     the series / Lentz continued fraction (Numerical Recipes sec. 6.2 formulation).
//   * 1-D quadrature: adaptive Gauss-Kronrod (7,15) bisection to the requested tolerance
//     (used for both the QNG and CQUAD entry points; only the accuracy contract matters,
//     the exact rule differs from GSL's, which is why construction parity with real-GSL
//     Agama is documented as unpinned at the ~1e-10 level).
//   * Brent's minimiser (golden section + parabolic interpolation, Brent 1973).
//   * Plain vector / matrix containers and simple linear fits.
// Everything else throws std::runtime_error("gsl shim: <name> not implemented").
#include "gsl/gsl_shim_all.h"
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>
#include <algorithm>

namespace {
[[noreturn]] void notImplemented(const char* name) {
    throw std::runtime_error(std::string("gsl shim: ") + name + " not implemented");
}
gsl_error_handler_t* g_handler = nullptr;
void raise(const char* reason, int code) {
    if(g_handler) g_handler(reason, __FILE__, __LINE__, code);
}
}

extern "C" {

const char* gsl_version = "1.16-shim";

gsl_error_handler_t* gsl_set_error_handler(gsl_error_handler_t* h) {
    gsl_error_handler_t* old = g_handler; g_handler = h; return old;
}

int gsl_fcmp(double x1, double x2, double epsilon) {
    // relative comparison with tolerance epsilon scaled by the larger exponent
    int exponent;
    double maxabs = std::fabs(x1) > std::fabs(x2) ? x1 : x2;
    std::frexp(maxabs, &exponent);
    double delta = std::ldexp(epsilon, exponent);
    double diff = x1 - x2;
    if(diff > delta) return 1;
    if(diff < -delta) return -1;
    return 0;
}

// ---------------- containers ----------------
gsl_vector* gsl_vector_alloc(size_t n) {
    gsl_vector* v = new gsl_vector;
    v->size = n; v->stride = 1; v->data = new double[n ? n : 1](); v->block = nullptr; v->owner = 1;
    return v;
}
void gsl_vector_free(gsl_vector* v) { if(!v) return; if(v->owner) delete[] v->data; delete v; }
double gsl_vector_get(const gsl_vector* v, size_t i) { return v->data[i * v->stride]; }
void gsl_vector_set(gsl_vector* v, size_t i, double x) { v->data[i * v->stride] = x; }
gsl_vector_view gsl_vector_view_array(double* base, size_t n) {
    gsl_vector_view w; w.vector.size = n; w.vector.stride = 1; w.vector.data = base;
    w.vector.block = nullptr; w.vector.owner = 0; return w;
}
gsl_vector_const_view gsl_vector_const_view_array(const double* base, size_t n) {
    gsl_vector_const_view w; w.vector.size = n; w.vector.stride = 1;
    w.vector.data = const_cast<double*>(base); w.vector.block = nullptr; w.vector.owner = 0; return w;
}
gsl_matrix* gsl_matrix_alloc(size_t n1, size_t n2) {
    gsl_matrix* m = new gsl_matrix;
    m->size1 = n1; m->size2 = n2; m->tda = n2; m->data = new double[n1 * n2 ? n1 * n2 : 1]();
    m->block = nullptr; m->owner = 1; return m;
}
void gsl_matrix_free(gsl_matrix* m) { if(!m) return; if(m->owner) delete[] m->data; delete m; }
double gsl_matrix_get(const gsl_matrix* m, size_t i, size_t j) { return m->data[i * m->tda + j]; }
void gsl_matrix_set(gsl_matrix* m, size_t i, size_t j, double x) { m->data[i * m->tda + j] = x; }
int gsl_matrix_memcpy(gsl_matrix* dest, const gsl_matrix* src) {
    if(dest->size1 != src->size1 || dest->size2 != src->size2) notImplemented("gsl_matrix_memcpy(size mismatch)");
    for(size_t i = 0; i < src->size1; i++)
        for(size_t j = 0; j < src->size2; j++)
            dest->data[i * dest->tda + j] = src->data[i * src->tda + j];
    return GSL_SUCCESS;
}
gsl_matrix_view gsl_matrix_view_array(double* base, size_t n1, size_t n2) {
    gsl_matrix_view v; v.matrix.size1 = n1; v.matrix.size2 = n2; v.matrix.tda = n2;
    v.matrix.data = base; v.matrix.block = nullptr; v.matrix.owner = 0; return v;
}
gsl_matrix_const_view gsl_matrix_const_view_array(const double* base, size_t n1, size_t n2) {
    gsl_matrix_const_view v; v.matrix.size1 = n1; v.matrix.size2 = n2; v.matrix.tda = n2;
    v.matrix.data = const_cast<double*>(base); v.matrix.block = nullptr; v.matrix.owner = 0; return v;
}
gsl_matrix_const_view gsl_matrix_const_submatrix(const gsl_matrix* m, size_t i, size_t j, size_t n1, size_t n2) {
    gsl_matrix_const_view v; v.matrix.size1 = n1; v.matrix.size2 = n2; v.matrix.tda = m->tda;
    v.matrix.data = m->data + i * m->tda + j; v.matrix.block = nullptr; v.matrix.owner = 0; return v;
}
gsl_permutation* gsl_permutation_alloc(size_t n) {
    gsl_permutation* p = new gsl_permutation; p->size = n; p->data = new size_t[n ? n : 1];
    for(size_t i = 0; i < n; i++) p->data[i] = i;
    return p;
}
void gsl_permutation_free(gsl_permutation* p) { if(!p) return; delete[] p->data; delete p; }
int gsl_permutation_memcpy(gsl_permutation* d, const gsl_permutation* s) {
    std::memcpy(d->data, s->data, s->size * sizeof(size_t)); return GSL_SUCCESS;
}

// ---------------- BLAS / linear algebra: not reached on the oracle paths ----------------
int gsl_blas_ddot(const gsl_vector* x, const gsl_vector* y, double* r) {
    double s = 0;
    for(size_t i = 0; i < x->size; i++) s += x->data[i * x->stride] * y->data[i * y->stride];
    *r = s; return GSL_SUCCESS;
}
int gsl_blas_dgemv(CBLAS_TRANSPOSE_t, double, const gsl_matrix*, const gsl_vector*, double, gsl_vector*)
{ notImplemented("gsl_blas_dgemv"); }
int gsl_blas_dgemm(CBLAS_TRANSPOSE_t, CBLAS_TRANSPOSE_t, double, const gsl_matrix*, const gsl_matrix*, double, gsl_matrix*)
{ notImplemented("gsl_blas_dgemm"); }
int gsl_blas_dtrsv(CBLAS_UPLO_t, CBLAS_TRANSPOSE_t, CBLAS_DIAG_t, const gsl_matrix*, gsl_vector*)
{ notImplemented("gsl_blas_dtrsv"); }
int gsl_blas_dtrmv(CBLAS_UPLO_t, CBLAS_TRANSPOSE_t, CBLAS_DIAG_t, const gsl_matrix*, gsl_vector*)
{ notImplemented("gsl_blas_dtrmv"); }
int gsl_blas_dtrsm(CBLAS_SIDE_t, CBLAS_UPLO_t, CBLAS_TRANSPOSE_t, CBLAS_DIAG_t, double, const gsl_matrix*, gsl_matrix*)
{ notImplemented("gsl_blas_dtrsm"); }
int gsl_linalg_LU_decomp(gsl_matrix*, gsl_permutation*, int*) { notImplemented("gsl_linalg_LU_decomp"); }
int gsl_linalg_LU_solve(const gsl_matrix*, const gsl_permutation*, const gsl_vector*, gsl_vector*)
{ notImplemented("gsl_linalg_LU_solve"); }
int gsl_linalg_cholesky_decomp(gsl_matrix*) { notImplemented("gsl_linalg_cholesky_decomp"); }
int gsl_linalg_cholesky_solve(const gsl_matrix*, const gsl_vector*, gsl_vector*)
{ notImplemented("gsl_linalg_cholesky_solve"); }
int gsl_linalg_QR_decomp(gsl_matrix*, gsl_vector*) { notImplemented("gsl_linalg_QR_decomp"); }
int gsl_linalg_QR_unpack(const gsl_matrix*, const gsl_vector*, gsl_matrix*, gsl_matrix*)
{ notImplemented("gsl_linalg_QR_unpack"); }
int gsl_linalg_QR_QTvec(const gsl_matrix*, const gsl_vector*, gsl_vector*) { notImplemented("gsl_linalg_QR_QTvec"); }
int gsl_linalg_SV_decomp(gsl_matrix*, gsl_matrix*, gsl_vector*, gsl_vector*) { notImplemented("gsl_linalg_SV_decomp"); }
int gsl_linalg_SV_decomp_mod(gsl_matrix*, gsl_matrix*, gsl_matrix*, gsl_vector*, gsl_vector*)
{ notImplemented("gsl_linalg_SV_decomp_mod"); }
int gsl_linalg_SV_solve(const gsl_matrix*, const gsl_matrix*, const gsl_vector*, const gsl_vector*, gsl_vector*)
{ notImplemented("gsl_linalg_SV_solve"); }

// ---------------- Brent minimiser ----------------
struct gsl_min_fminimizer_s {
    gsl_function* f;
    double x, fx, a, fa, b, fb;   // current best point and bracket
    double v, fv, w, fw;          // previous best points
    double d, e;                  // last and second-to-last steps
};
static const gsl_min_fminimizer_type brentType = { "brent" };
const gsl_min_fminimizer_type* gsl_min_fminimizer_brent = &brentType;

gsl_min_fminimizer* gsl_min_fminimizer_alloc(const gsl_min_fminimizer_type*) { return new gsl_min_fminimizer_s(); }
void gsl_min_fminimizer_free(gsl_min_fminimizer* s) { delete s; }
int gsl_min_fminimizer_set_with_values(gsl_min_fminimizer* s, gsl_function* f,
    double xm, double fm, double xl, double fl, double xu, double fu)
{
    if(!(xl < xm && xm < xu) || !(fm < fl && fm < fu)) {
        raise("minimum not bracketed", GSL_EINVAL);
        return GSL_EINVAL;
    }
    s->f = f; s->x = xm; s->fx = fm; s->a = xl; s->fa = fl; s->b = xu; s->fb = fu;
    const double golden = 0.3819660112501051;
    s->v = xl + golden * (xu - xl);
    s->fv = f->function(s->v, f->params);
    s->w = s->v; s->fw = s->fv; s->d = 0; s->e = 0;
    return GSL_SUCCESS;
}
int gsl_min_fminimizer_iterate(gsl_min_fminimizer* s) {
    // one step of Brent's method: parabolic interpolation through (v, w, x) when it is
    // acceptable, otherwise a golden-section step into the larger sub-interval
    const double golden = 0.3819660112501051;
    const double tol = 1.4901161193847656e-08 * std::fabs(s->x) + 1e-10;
    double mid = 0.5 * (s->a + s->b), u, step;
    bool parabolic = false;
    if(std::fabs(s->e) > tol) {
        double r = (s->x - s->w) * (s->fx - s->fv);
        double q = (s->x - s->v) * (s->fx - s->fw);
        double p = (s->x - s->v) * q - (s->x - s->w) * r;
        q = 2 * (q - r);
        if(q > 0) p = -p; else q = -q;
        if(std::fabs(p) < std::fabs(0.5 * q * s->e) && p > q * (s->a - s->x) && p < q * (s->b - s->x)) {
            step = p / q;
            u = s->x + step;
            if(u - s->a < 2 * tol || s->b - u < 2 * tol) step = s->x < mid ? tol : -tol;
            parabolic = true;
        }
    }
    if(!parabolic) {
        s->e = (s->x < mid ? s->b : s->a) - s->x;
        step = golden * s->e;
    } else {
        s->e = s->d;
    }
    s->d = step;
    u = std::fabs(step) >= tol ? s->x + step : s->x + (step > 0 ? tol : -tol);
    double fu = s->f->function(u, s->f->params);
    if(!std::isfinite(fu)) { raise("function not finite", GSL_EBADFUNC); return GSL_EBADFUNC; }
    if(fu <= s->fx) {
        if(u < s->x) { s->b = s->x; s->fb = s->fx; } else { s->a = s->x; s->fa = s->fx; }
        s->v = s->w; s->fv = s->fw; s->w = s->x; s->fw = s->fx; s->x = u; s->fx = fu;
    } else {
        if(u < s->x) { s->a = u; s->fa = fu; } else { s->b = u; s->fb = fu; }
        if(fu <= s->fw || s->w == s->x) { s->v = s->w; s->fv = s->fw; s->w = u; s->fw = fu; }
        else if(fu <= s->fv || s->v == s->x || s->v == s->w) { s->v = u; s->fv = fu; }
    }
    return GSL_SUCCESS;
}
double gsl_min_fminimizer_x_minimum(const gsl_min_fminimizer* s) { return s->x; }
double gsl_min_fminimizer_x_lower(const gsl_min_fminimizer* s) { return s->a; }
double gsl_min_fminimizer_x_upper(const gsl_min_fminimizer* s) { return s->b; }

// ---------------- adaptive Gauss-Kronrod quadrature ----------------
namespace {
// nodes and weights of the 15-point Kronrod extension of the 7-point Gauss rule on [-1,1]
const double XGK[8] = { 0.991455371120812639206854697526329, 0.949107912342758524526189684047851,
    0.864864423359769072789712788640926, 0.741531185599394439863864773280788,
    0.586087235467691130294144845693013, 0.405845151377397166906606412076961,
    0.207784955007898467600689403773245, 0.0 };
const double WGK[8] = { 0.022935322010529224963732008058970, 0.063092092629978553290700663189204,
    0.104790010322250183839876322541518, 0.140653259715525918745189590510238,
    0.169004726639267902826583426598550, 0.190350578064785409913256402421014,
    0.204432940075298892414161999234649, 0.209482141084727828012999174891714 };
const double WG[4] = { 0.129484966168869693270611432679082, 0.279705391489276667901467771423780,
    0.381830050505118944950369775488975, 0.417959183673469387755102040816327 };

struct Segment { double a, b, val, err; };

Segment gk15(const gsl_function* f, double a, double b, size_t& neval) {
    double c = 0.5 * (a + b), h = 0.5 * (b - a);
    double fc = f->function(c, f->params);
    double resk = fc * WGK[7], resg = fc * WG[3];
    for(int j = 0; j < 7; j++) {
        double dx = h * XGK[j];
        double f1 = f->function(c - dx, f->params), f2 = f->function(c + dx, f->params);
        resk += WGK[j] * (f1 + f2);
        if(j % 2 == 1) resg += WG[j / 2] * (f1 + f2);
    }
    neval += 15;
    Segment s; s.a = a; s.b = b; s.val = resk * h; s.err = std::fabs((resk - resg) * h);
    return s;
}

int adaptive(const gsl_function* f, double a, double b, double epsabs, double epsrel,
    double* result, double* abserr, size_t* neval, size_t maxseg)
{
    size_t count = 0;
    std::vector<Segment> segs(1, gk15(f, a, b, count));
    double total = segs[0].val, toterr = segs[0].err;
    while(toterr > std::max(epsabs, epsrel * std::fabs(total)) && segs.size() < maxseg) {
        size_t worst = 0;
        for(size_t i = 1; i < segs.size(); i++) if(segs[i].err > segs[worst].err) worst = i;
        Segment s = segs[worst];
        double mid = 0.5 * (s.a + s.b);
        if(!(mid > std::min(s.a, s.b) && mid < std::max(s.a, s.b))) break;  // cannot subdivide further
        Segment l = gk15(f, s.a, mid, count), r = gk15(f, mid, s.b, count);
        segs[worst] = l; segs.push_back(r);
        total = 0; toterr = 0;
        for(size_t i = 0; i < segs.size(); i++) { total += segs[i].val; toterr += segs[i].err; }
    }
    *result = total;
    if(abserr) *abserr = toterr;
    if(neval) *neval = count;
    if(!std::isfinite(total)) { raise("integrand not finite", GSL_EDIVERGE); return GSL_EDIVERGE; }
    return GSL_SUCCESS;
}
}  // namespace

struct gsl_integration_cquad_workspace_s { size_t n; };
int gsl_integration_qng(const gsl_function* f, double a, double b, double epsabs, double epsrel,
    double* result, double* abserr, size_t* neval)
{ return adaptive(f, a, b, epsabs, epsrel, result, abserr, neval, 64); }
gsl_integration_cquad_workspace* gsl_integration_cquad_workspace_alloc(size_t n) {
    gsl_integration_cquad_workspace* w = new gsl_integration_cquad_workspace_s; w->n = n; return w;
}
void gsl_integration_cquad_workspace_free(gsl_integration_cquad_workspace* w) { delete w; }
int gsl_integration_cquad(const gsl_function* f, double a, double b, double epsabs, double epsrel,
    gsl_integration_cquad_workspace* ws, double* result, double* abserr, size_t* nevals)
{ return adaptive(f, a, b, epsabs, epsrel, result, abserr, nevals, ws ? ws->n : 1000); }

// ---------------- special functions ----------------
double gsl_sf_gamma(double x) { return std::tgamma(x); }
double gsl_sf_lngamma(double x) { return std::lgamma(x); }
double gsl_sf_gamma_inc(double a, double x) {
    // non-normalised upper incomplete gamma  Gamma(a,x) = Gamma(a) Q(a,x),  a>0, x>=0
    if(!(a > 0) || !(x >= 0)) notImplemented("gsl_sf_gamma_inc(a<=0 or x<0)");
    if(x == 0) return std::tgamma(a);
    double lnpre = a * std::log(x) - x - std::lgamma(a);
    double Q;
    if(x < a + 1) {   // series for P(a,x)
        double sum = 1 / a, term = sum;
        for(int n = 1; n < 1000; n++) {
            term *= x / (a + n); sum += term;
            if(std::fabs(term) < std::fabs(sum) * 1e-17) break;
        }
        Q = 1 - sum * std::exp(lnpre);
    } else {          // modified Lentz continued fraction for Q(a,x)
        const double tiny = 1e-300;
        double b = x + 1 - a, c = 1 / tiny, d = 1 / b, h = d;
        for(int i = 1; i < 1000; i++) {
            double an = -i * (i - a);
            b += 2;
            d = an * d + b; if(std::fabs(d) < tiny) d = tiny;
            c = b + an / c; if(std::fabs(c) < tiny) c = tiny;
            d = 1 / d;
            double del = d * c; h *= del;
            if(std::fabs(del - 1) < 1e-16) break;
        }
        Q = std::exp(lnpre) * h;
    }
    return Q * std::tgamma(a);
}
double gsl_sf_fact(unsigned int n) { return std::tgamma(n + 1.0); }
double gsl_sf_lnfact(unsigned int n) { return std::lgamma(n + 1.0); }
double gsl_sf_doublefact(unsigned int n) {
    double r = 1; for(unsigned int k = n; k > 1; k -= 2) r *= k; return r;
}
double gsl_sf_psi(double) { notImplemented("gsl_sf_psi"); }
double gsl_sf_psi_int(int) { notImplemented("gsl_sf_psi_int"); }
double gsl_sf_hyperg_2F1(double, double, double, double) { notImplemented("gsl_sf_hyperg_2F1"); }
double gsl_sf_ellint_Kcomp(double, gsl_mode_t) { notImplemented("gsl_sf_ellint_Kcomp"); }
double gsl_sf_ellint_Ecomp(double, gsl_mode_t) { notImplemented("gsl_sf_ellint_Ecomp"); }
double gsl_sf_ellint_F(double, double, gsl_mode_t) { notImplemented("gsl_sf_ellint_F"); }
double gsl_sf_ellint_E(double, double, gsl_mode_t) { notImplemented("gsl_sf_ellint_E"); }
double gsl_sf_ellint_P(double, double, double, gsl_mode_t) { notImplemented("gsl_sf_ellint_P"); }
double gsl_sf_bessel_Jn(int, double) { notImplemented("gsl_sf_bessel_Jn"); }
double gsl_sf_bessel_Yn(int, double) { notImplemented("gsl_sf_bessel_Yn"); }
double gsl_sf_bessel_In(int, double) { notImplemented("gsl_sf_bessel_In"); }
double gsl_sf_bessel_Kn(int, double) { notImplemented("gsl_sf_bessel_Kn"); }

static double lambertHalley(double x, double w) {
    // Halley iteration for w e^w = x
    for(int i = 0; i < 100; i++) {
        double ew = std::exp(w), f = w * ew - x;
        double wp1 = w + 1;
        double denom = ew * wp1 - (w + 2) * f / (2 * wp1);
        double dw = f / denom;
        w -= dw;
        if(std::fabs(dw) <= 4e-16 * (1 + std::fabs(w))) break;
    }
    return w;
}
double gsl_sf_lambert_W0(double x) {
    const double branchPoint = -0.36787944117144233;  // -1/e
    if(x < branchPoint) return NAN;
    if(x == 0) return 0;
    if(x == branchPoint) return -1;
    double w;
    if(x < -0.25) {   // series around the branch point in p = sqrt(2(e x + 1))
        double p = std::sqrt(2 * (2.718281828459045 * x + 1));
        w = -1 + p - p * p / 3 + 11. / 72 * p * p * p;
    } else if(x < 3) w = std::log1p(x) * (1 - std::log1p(std::log1p(x)) / (2 + std::log1p(x)));
    else { double l1 = std::log(x), l2 = std::log(l1); w = l1 - l2 + l2 / l1; }
    return lambertHalley(x, w);
}
double gsl_sf_lambert_Wm1(double x) {
    const double branchPoint = -0.36787944117144233;
    if(x < branchPoint || x >= 0) return x == 0 ? -INFINITY : NAN;
    if(x == branchPoint) return -1;
    double w;
    if(x < -0.25) {
        double p = -std::sqrt(2 * (2.718281828459045 * x + 1));
        w = -1 + p - p * p / 3 + 11. / 72 * p * p * p;
    } else { double l1 = std::log(-x), l2 = std::log(-l1); w = l1 - l2 + l2 / l1; }
    return lambertHalley(x, w);
}

// ---------------- linear fits ----------------
int gsl_fit_wlinear(const double* x, size_t xs, const double* w, size_t ws, const double* y, size_t ys,
    size_t n, double* c0, double* c1, double* cov00, double* cov01, double* cov11, double* chisq)
{
    double W = 0, wx = 0, wy = 0;
    for(size_t i = 0; i < n; i++) {
        double wi = w ? w[i * ws] : 1; W += wi; wx += wi * x[i * xs]; wy += wi * y[i * ys];
    }
    wx /= W; wy /= W;
    double dxx = 0, dxy = 0;
    for(size_t i = 0; i < n; i++) {
        double wi = w ? w[i * ws] : 1, dx = x[i * xs] - wx, dy = y[i * ys] - wy;
        dxx += wi * dx * dx; dxy += wi * dx * dy;
    }
    double b = dxy / dxx, a = wy - wx * b, d2 = 0;
    for(size_t i = 0; i < n; i++) {
        double wi = w ? w[i * ws] : 1, r = y[i * ys] - (a + b * x[i * xs]); d2 += wi * r * r;
    }
    *c0 = a; *c1 = b;
    double s2 = w ? 1 : d2 / (n > 2 ? n - 2 : 1);
    *cov00 = s2 * (1 / W) * (1 + wx * wx / (dxx / W));
    *cov11 = s2 / dxx;
    *cov01 = -s2 * wx / dxx;
    *chisq = d2;
    return GSL_SUCCESS;
}
int gsl_fit_linear(const double* x, size_t xs, const double* y, size_t ys, size_t n,
    double* c0, double* c1, double* cov00, double* cov01, double* cov11, double* sumsq)
{ return gsl_fit_wlinear(x, xs, nullptr, 0, y, ys, n, c0, c1, cov00, cov01, cov11, sumsq); }
int gsl_fit_wmul(const double* x, size_t xs, const double* w, size_t ws, const double* y, size_t ys,
    size_t n, double* c1, double* cov11, double* sumsq)
{
    double sxx = 0, sxy = 0;
    for(size_t i = 0; i < n; i++) {
        double wi = w ? w[i * ws] : 1; sxx += wi * x[i * xs] * x[i * xs]; sxy += wi * x[i * xs] * y[i * ys];
    }
    double b = sxy / sxx, d2 = 0;
    for(size_t i = 0; i < n; i++) {
        double wi = w ? w[i * ws] : 1, r = y[i * ys] - b * x[i * xs]; d2 += wi * r * r;
    }
    *c1 = b; *cov11 = (w ? 1 : d2 / (n > 1 ? n - 1 : 1)) / sxx; *sumsq = d2;
    return GSL_SUCCESS;
}
int gsl_fit_mul(const double* x, size_t xs, const double* y, size_t ys, size_t n,
    double* c1, double* cov11, double* sumsq)
{ return gsl_fit_wmul(x, xs, nullptr, 0, y, ys, n, c1, cov11, sumsq); }

// ---------------- not reached: multi-dimensional fitting / roots / minimisation ----------------
gsl_multifit_linear_workspace* gsl_multifit_linear_alloc(size_t, size_t) { notImplemented("gsl_multifit_linear_alloc"); }
void gsl_multifit_linear_free(gsl_multifit_linear_workspace*) {}
int gsl_multifit_linear(const gsl_matrix*, const gsl_vector*, gsl_vector*, gsl_matrix*, double*,
    gsl_multifit_linear_workspace*) { notImplemented("gsl_multifit_linear"); }
int gsl_multifit_wlinear(const gsl_matrix*, const gsl_vector*, const gsl_vector*, gsl_vector*,
    gsl_matrix*, double*, gsl_multifit_linear_workspace*) { notImplemented("gsl_multifit_wlinear"); }
static const gsl_multifit_fdfsolver_type lmsderType = { "lmsder" };
const gsl_multifit_fdfsolver_type* gsl_multifit_fdfsolver_lmsder = &lmsderType;
gsl_multifit_fdfsolver* gsl_multifit_fdfsolver_alloc(const gsl_multifit_fdfsolver_type*, size_t, size_t)
{ notImplemented("gsl_multifit_fdfsolver_alloc"); }
int gsl_multifit_fdfsolver_set(gsl_multifit_fdfsolver*, gsl_multifit_function_fdf*, const gsl_vector*)
{ notImplemented("gsl_multifit_fdfsolver_set"); }
int gsl_multifit_fdfsolver_iterate(gsl_multifit_fdfsolver*) { notImplemented("gsl_multifit_fdfsolver_iterate"); }
void gsl_multifit_fdfsolver_free(gsl_multifit_fdfsolver*) {}
int gsl_multifit_test_delta(const gsl_vector*, const gsl_vector*, double, double)
{ notImplemented("gsl_multifit_test_delta"); }
static const gsl_multiroot_fdfsolver_type hybridsjType = { "hybridsj" };
const gsl_multiroot_fdfsolver_type* gsl_multiroot_fdfsolver_hybridsj = &hybridsjType;
gsl_multiroot_fdfsolver* gsl_multiroot_fdfsolver_alloc(const gsl_multiroot_fdfsolver_type*, size_t)
{ notImplemented("gsl_multiroot_fdfsolver_alloc"); }
int gsl_multiroot_fdfsolver_set(gsl_multiroot_fdfsolver*, gsl_multiroot_function_fdf*, const gsl_vector*)
{ notImplemented("gsl_multiroot_fdfsolver_set"); }
int gsl_multiroot_fdfsolver_iterate(gsl_multiroot_fdfsolver*) { notImplemented("gsl_multiroot_fdfsolver_iterate"); }
void gsl_multiroot_fdfsolver_free(gsl_multiroot_fdfsolver*) {}
int gsl_multiroot_test_residual(const gsl_vector*, double) { notImplemented("gsl_multiroot_test_residual"); }
int gsl_multiroot_test_delta(const gsl_vector*, const gsl_vector*, double, double)
{ notImplemented("gsl_multiroot_test_delta"); }
static const gsl_multimin_fminimizer_type nmType = { "nmsimplex2" };
static const gsl_multimin_fdfminimizer_type bfgsType = { "vector_bfgs2" };
const gsl_multimin_fminimizer_type* gsl_multimin_fminimizer_nmsimplex2 = &nmType;
const gsl_multimin_fdfminimizer_type* gsl_multimin_fdfminimizer_vector_bfgs2 = &bfgsType;
gsl_multimin_fminimizer* gsl_multimin_fminimizer_alloc(const gsl_multimin_fminimizer_type*, size_t)
{ notImplemented("gsl_multimin_fminimizer_alloc"); }
int gsl_multimin_fminimizer_set(gsl_multimin_fminimizer*, gsl_multimin_function*, const gsl_vector*, const gsl_vector*)
{ notImplemented("gsl_multimin_fminimizer_set"); }
int gsl_multimin_fminimizer_iterate(gsl_multimin_fminimizer*) { notImplemented("gsl_multimin_fminimizer_iterate"); }
double gsl_multimin_fminimizer_size(const gsl_multimin_fminimizer*) { notImplemented("gsl_multimin_fminimizer_size"); }
void gsl_multimin_fminimizer_free(gsl_multimin_fminimizer*) {}
gsl_multimin_fdfminimizer* gsl_multimin_fdfminimizer_alloc(const gsl_multimin_fdfminimizer_type*, size_t)
{ notImplemented("gsl_multimin_fdfminimizer_alloc"); }
int gsl_multimin_fdfminimizer_set(gsl_multimin_fdfminimizer*, gsl_multimin_function_fdf*, const gsl_vector*, double, double)
{ notImplemented("gsl_multimin_fdfminimizer_set"); }
int gsl_multimin_fdfminimizer_iterate(gsl_multimin_fdfminimizer*) { notImplemented("gsl_multimin_fdfminimizer_iterate"); }
void gsl_multimin_fdfminimizer_free(gsl_multimin_fdfminimizer*) {}
int gsl_multimin_test_gradient(const gsl_vector*, double) { notImplemented("gsl_multimin_test_gradient"); }

}  // extern "C"
