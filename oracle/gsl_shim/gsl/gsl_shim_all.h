/* Minimal stand-in for the GNU Scientific Library API, written for this project.

   TEST INFRASTRUCTURE ONLY: it exists so that the reference Agama sources can be
   compiled here (GSL is not installed and cannot be fetched) to serve as the CPU
   oracle.  Only declarations are provided in this header; gsl_shim.cpp implements
   the handful of functions that the Multipole construction, the density models of
   the benchmark configurations and the Staeckel-fudge set-up actually reach
   (Lambert W, Gamma, incomplete Gamma, 1-D adaptive quadrature, Brent minimiser).
   Every other entry point throws std::runtime_error("gsl shim: <name> ..."), so an
   unexpected use is loud rather than silently wrong.

   No GSL source code is used; the struct layouts mirror the documented public API
   so that the reference sources compile unchanged. */
#pragma once
#include <stddef.h>
#include <math.h>   /* the real headers pull these in transitively; the reference relies on it */
#include <float.h>

#define GSL_MAJOR_VERSION 1
#define GSL_MINOR_VERSION 16

#ifdef __cplusplus
extern "C" {
#endif

extern const char* gsl_version;

/* ---- error codes (gsl_errno.h) ---- */
enum {
    GSL_SUCCESS = 0, GSL_FAILURE = -1, GSL_CONTINUE = -2, GSL_EDOM = 1, GSL_ERANGE = 2,
    GSL_EFAULT = 3, GSL_EINVAL = 4, GSL_EFAILED = 5, GSL_EFACTOR = 6, GSL_ESANITY = 7,
    GSL_ENOMEM = 8, GSL_EBADFUNC = 9, GSL_ERUNAWAY = 10, GSL_EMAXITER = 11, GSL_EZERODIV = 12,
    GSL_EBADTOL = 13, GSL_ETOL = 14, GSL_EUNDRFLW = 15, GSL_EOVRFLW = 16, GSL_ELOSS = 17,
    GSL_EROUND = 18, GSL_EBADLEN = 19, GSL_ENOTSQR = 20, GSL_ESING = 21, GSL_EDIVERGE = 22,
    GSL_EUNSUP = 23, GSL_EUNIMPL = 24, GSL_ECACHE = 25, GSL_ETABLE = 26, GSL_ENOPROG = 27,
    GSL_ENOPROGJ = 28, GSL_ETOLF = 29, GSL_ETOLX = 30, GSL_ETOLG = 31, GSL_EOF = 32
};
typedef void gsl_error_handler_t(const char* reason, const char* file, int line, int gsl_errno);
gsl_error_handler_t* gsl_set_error_handler(gsl_error_handler_t* new_handler);

/* ---- precision mode (gsl_mode.h) ---- */
typedef unsigned int gsl_mode_t;
#define GSL_PREC_DOUBLE 0
#define GSL_PREC_SINGLE 1
#define GSL_PREC_APPROX 2

/* ---- math (gsl_math.h) ---- */
typedef struct { double (*function)(double x, void* params); void* params; } gsl_function;
int gsl_fcmp(double x1, double x2, double epsilon);

/* ---- blocks, vectors, matrices, permutations ---- */
typedef struct { size_t size; double* data; } gsl_block;
typedef struct { size_t size; size_t stride; double* data; gsl_block* block; int owner; } gsl_vector;
typedef struct { gsl_vector vector; } gsl_vector_view;
typedef struct { gsl_vector vector; } gsl_vector_const_view;
typedef struct { size_t size1; size_t size2; size_t tda; double* data; gsl_block* block; int owner; } gsl_matrix;
typedef struct { gsl_matrix matrix; } gsl_matrix_view;
typedef struct { gsl_matrix matrix; } gsl_matrix_const_view;
typedef struct { size_t size; size_t* data; } gsl_permutation;

gsl_vector* gsl_vector_alloc(size_t n);
void gsl_vector_free(gsl_vector* v);
double gsl_vector_get(const gsl_vector* v, size_t i);
void gsl_vector_set(gsl_vector* v, size_t i, double x);
gsl_vector_view gsl_vector_view_array(double* base, size_t n);
gsl_vector_const_view gsl_vector_const_view_array(const double* base, size_t n);
gsl_matrix* gsl_matrix_alloc(size_t n1, size_t n2);
void gsl_matrix_free(gsl_matrix* m);
double gsl_matrix_get(const gsl_matrix* m, size_t i, size_t j);
void gsl_matrix_set(gsl_matrix* m, size_t i, size_t j, double x);
int gsl_matrix_memcpy(gsl_matrix* dest, const gsl_matrix* src);
gsl_matrix_view gsl_matrix_view_array(double* base, size_t n1, size_t n2);
gsl_matrix_const_view gsl_matrix_const_view_array(const double* base, size_t n1, size_t n2);
gsl_matrix_const_view gsl_matrix_const_submatrix(const gsl_matrix* m, size_t i, size_t j, size_t n1, size_t n2);
gsl_permutation* gsl_permutation_alloc(size_t n);
void gsl_permutation_free(gsl_permutation* p);
int gsl_permutation_memcpy(gsl_permutation* dest, const gsl_permutation* src);

/* ---- BLAS (gsl_blas.h) ---- */
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
enum CBLAS_UPLO { CblasUpper = 121, CblasLower = 122 };
enum CBLAS_DIAG { CblasNonUnit = 131, CblasUnit = 132 };
enum CBLAS_SIDE { CblasLeft = 141, CblasRight = 142 };
typedef enum CBLAS_TRANSPOSE CBLAS_TRANSPOSE_t;
typedef enum CBLAS_UPLO CBLAS_UPLO_t;
typedef enum CBLAS_DIAG CBLAS_DIAG_t;
typedef enum CBLAS_SIDE CBLAS_SIDE_t;
int gsl_blas_ddot(const gsl_vector* x, const gsl_vector* y, double* result);
int gsl_blas_dgemv(CBLAS_TRANSPOSE_t TransA, double alpha, const gsl_matrix* A, const gsl_vector* x,
    double beta, gsl_vector* y);
int gsl_blas_dgemm(CBLAS_TRANSPOSE_t TransA, CBLAS_TRANSPOSE_t TransB, double alpha,
    const gsl_matrix* A, const gsl_matrix* B, double beta, gsl_matrix* C);
int gsl_blas_dtrsv(CBLAS_UPLO_t Uplo, CBLAS_TRANSPOSE_t TransA, CBLAS_DIAG_t Diag,
    const gsl_matrix* A, gsl_vector* X);
int gsl_blas_dtrmv(CBLAS_UPLO_t Uplo, CBLAS_TRANSPOSE_t TransA, CBLAS_DIAG_t Diag,
    const gsl_matrix* A, gsl_vector* X);
int gsl_blas_dtrsm(CBLAS_SIDE_t Side, CBLAS_UPLO_t Uplo, CBLAS_TRANSPOSE_t TransA, CBLAS_DIAG_t Diag,
    double alpha, const gsl_matrix* A, gsl_matrix* B);

/* ---- linear algebra (gsl_linalg.h) ---- */
int gsl_linalg_LU_decomp(gsl_matrix* A, gsl_permutation* p, int* signum);
int gsl_linalg_LU_solve(const gsl_matrix* LU, const gsl_permutation* p, const gsl_vector* b, gsl_vector* x);
int gsl_linalg_cholesky_decomp(gsl_matrix* A);
int gsl_linalg_cholesky_solve(const gsl_matrix* cholesky, const gsl_vector* b, gsl_vector* x);
int gsl_linalg_QR_decomp(gsl_matrix* A, gsl_vector* tau);
int gsl_linalg_QR_unpack(const gsl_matrix* QR, const gsl_vector* tau, gsl_matrix* Q, gsl_matrix* R);
int gsl_linalg_QR_QTvec(const gsl_matrix* QR, const gsl_vector* tau, gsl_vector* v);
int gsl_linalg_SV_decomp(gsl_matrix* A, gsl_matrix* V, gsl_vector* S, gsl_vector* work);
int gsl_linalg_SV_decomp_mod(gsl_matrix* A, gsl_matrix* X, gsl_matrix* V, gsl_vector* S, gsl_vector* work);
int gsl_linalg_SV_solve(const gsl_matrix* U, const gsl_matrix* V, const gsl_vector* S,
    const gsl_vector* b, gsl_vector* x);

/* ---- 1-D minimisation (gsl_min.h) ---- */
typedef struct gsl_min_fminimizer_type_s { const char* name; } gsl_min_fminimizer_type;
typedef struct gsl_min_fminimizer_s gsl_min_fminimizer;
extern const gsl_min_fminimizer_type* gsl_min_fminimizer_brent;
gsl_min_fminimizer* gsl_min_fminimizer_alloc(const gsl_min_fminimizer_type* T);
void gsl_min_fminimizer_free(gsl_min_fminimizer* s);
int gsl_min_fminimizer_set_with_values(gsl_min_fminimizer* s, gsl_function* f,
    double x_minimum, double f_minimum, double x_lower, double f_lower, double x_upper, double f_upper);
int gsl_min_fminimizer_iterate(gsl_min_fminimizer* s);
double gsl_min_fminimizer_x_minimum(const gsl_min_fminimizer* s);
double gsl_min_fminimizer_x_lower(const gsl_min_fminimizer* s);
double gsl_min_fminimizer_x_upper(const gsl_min_fminimizer* s);

/* ---- 1-D integration (gsl_integration.h) ---- */
typedef struct gsl_integration_cquad_workspace_s gsl_integration_cquad_workspace;
int gsl_integration_qng(const gsl_function* f, double a, double b, double epsabs, double epsrel,
    double* result, double* abserr, size_t* neval);
gsl_integration_cquad_workspace* gsl_integration_cquad_workspace_alloc(size_t n);
void gsl_integration_cquad_workspace_free(gsl_integration_cquad_workspace* w);
int gsl_integration_cquad(const gsl_function* f, double a, double b, double epsabs, double epsrel,
    gsl_integration_cquad_workspace* ws, double* result, double* abserr, size_t* nevals);

/* ---- special functions (gsl_sf_*.h) ---- */
double gsl_sf_gamma(double x);
double gsl_sf_lngamma(double x);
double gsl_sf_gamma_inc(double a, double x);
double gsl_sf_fact(unsigned int n);
double gsl_sf_lnfact(unsigned int n);
double gsl_sf_doublefact(unsigned int n);
double gsl_sf_psi(double x);
double gsl_sf_psi_int(int n);
double gsl_sf_hyperg_2F1(double a, double b, double c, double x);
double gsl_sf_ellint_Kcomp(double k, gsl_mode_t mode);
double gsl_sf_ellint_Ecomp(double k, gsl_mode_t mode);
double gsl_sf_ellint_F(double phi, double k, gsl_mode_t mode);
double gsl_sf_ellint_E(double phi, double k, gsl_mode_t mode);
double gsl_sf_ellint_P(double phi, double k, double n, gsl_mode_t mode);
double gsl_sf_bessel_Jn(int n, double x);
double gsl_sf_bessel_Yn(int n, double x);
double gsl_sf_bessel_In(int n, double x);
double gsl_sf_bessel_Kn(int n, double x);
double gsl_sf_lambert_W0(double x);
double gsl_sf_lambert_Wm1(double x);

/* ---- linear fits (gsl_fit.h) ---- */
int gsl_fit_linear(const double* x, size_t xstride, const double* y, size_t ystride, size_t n,
    double* c0, double* c1, double* cov00, double* cov01, double* cov11, double* sumsq);
int gsl_fit_wlinear(const double* x, size_t xstride, const double* w, size_t wstride,
    const double* y, size_t ystride, size_t n,
    double* c0, double* c1, double* cov00, double* cov01, double* cov11, double* chisq);
int gsl_fit_mul(const double* x, size_t xstride, const double* y, size_t ystride, size_t n,
    double* c1, double* cov11, double* sumsq);
int gsl_fit_wmul(const double* x, size_t xstride, const double* w, size_t wstride,
    const double* y, size_t ystride, size_t n, double* c1, double* cov11, double* sumsq);

/* ---- multi-parameter linear fits (gsl_multifit.h) ---- */
typedef struct gsl_multifit_linear_workspace_s gsl_multifit_linear_workspace;
gsl_multifit_linear_workspace* gsl_multifit_linear_alloc(size_t n, size_t p);
void gsl_multifit_linear_free(gsl_multifit_linear_workspace* w);
int gsl_multifit_linear(const gsl_matrix* X, const gsl_vector* y, gsl_vector* c, gsl_matrix* cov,
    double* chisq, gsl_multifit_linear_workspace* work);
int gsl_multifit_wlinear(const gsl_matrix* X, const gsl_vector* w, const gsl_vector* y, gsl_vector* c,
    gsl_matrix* cov, double* chisq, gsl_multifit_linear_workspace* work);

/* ---- nonlinear least squares (gsl_multifit_nlin.h) ---- */
typedef struct {
    int (*f)(const gsl_vector* x, void* params, gsl_vector* f);
    int (*df)(const gsl_vector* x, void* params, gsl_matrix* df);
    int (*fdf)(const gsl_vector* x, void* params, gsl_vector* f, gsl_matrix* df);
    size_t n; size_t p; void* params;
} gsl_multifit_function_fdf;
typedef struct { const char* name; } gsl_multifit_fdfsolver_type;
typedef struct { const gsl_multifit_fdfsolver_type* type; gsl_multifit_function_fdf* fdf;
    gsl_vector* x; gsl_vector* f; gsl_matrix* J; gsl_vector* dx; void* state; } gsl_multifit_fdfsolver;
extern const gsl_multifit_fdfsolver_type* gsl_multifit_fdfsolver_lmsder;
gsl_multifit_fdfsolver* gsl_multifit_fdfsolver_alloc(const gsl_multifit_fdfsolver_type* T, size_t n, size_t p);
int gsl_multifit_fdfsolver_set(gsl_multifit_fdfsolver* s, gsl_multifit_function_fdf* fdf, const gsl_vector* x);
int gsl_multifit_fdfsolver_iterate(gsl_multifit_fdfsolver* s);
void gsl_multifit_fdfsolver_free(gsl_multifit_fdfsolver* s);
int gsl_multifit_test_delta(const gsl_vector* dx, const gsl_vector* x, double epsabs, double epsrel);

/* ---- multidimensional root finding (gsl_multiroots.h) ---- */
typedef struct {
    int (*f)(const gsl_vector* x, void* params, gsl_vector* f);
    int (*df)(const gsl_vector* x, void* params, gsl_matrix* df);
    int (*fdf)(const gsl_vector* x, void* params, gsl_vector* f, gsl_matrix* df);
    size_t n; void* params;
} gsl_multiroot_function_fdf;
typedef struct { const char* name; } gsl_multiroot_fdfsolver_type;
typedef struct { const gsl_multiroot_fdfsolver_type* type; gsl_multiroot_function_fdf* fdf;
    gsl_vector* x; gsl_vector* f; gsl_matrix* J; gsl_vector* dx; void* state; } gsl_multiroot_fdfsolver;
extern const gsl_multiroot_fdfsolver_type* gsl_multiroot_fdfsolver_hybridsj;
gsl_multiroot_fdfsolver* gsl_multiroot_fdfsolver_alloc(const gsl_multiroot_fdfsolver_type* T, size_t n);
int gsl_multiroot_fdfsolver_set(gsl_multiroot_fdfsolver* s, gsl_multiroot_function_fdf* fdf, const gsl_vector* x);
int gsl_multiroot_fdfsolver_iterate(gsl_multiroot_fdfsolver* s);
void gsl_multiroot_fdfsolver_free(gsl_multiroot_fdfsolver* s);
int gsl_multiroot_test_residual(const gsl_vector* f, double epsabs);
int gsl_multiroot_test_delta(const gsl_vector* dx, const gsl_vector* x, double epsabs, double epsrel);

/* ---- multidimensional minimisation (gsl_multimin.h) ---- */
typedef struct { double (*f)(const gsl_vector* x, void* params); size_t n; void* params; } gsl_multimin_function;
typedef struct {
    double (*f)(const gsl_vector* x, void* params);
    void (*df)(const gsl_vector* x, void* params, gsl_vector* df);
    void (*fdf)(const gsl_vector* x, void* params, double* f, gsl_vector* df);
    size_t n; void* params;
} gsl_multimin_function_fdf;
typedef struct { const char* name; } gsl_multimin_fminimizer_type;
typedef struct { const char* name; } gsl_multimin_fdfminimizer_type;
typedef struct { const gsl_multimin_fminimizer_type* type; gsl_multimin_function* f;
    double fval; gsl_vector* x; double size; void* state; } gsl_multimin_fminimizer;
typedef struct { const gsl_multimin_fdfminimizer_type* type; gsl_multimin_function_fdf* fdf;
    double f; gsl_vector* x; gsl_vector* gradient; gsl_vector* dx; void* state; } gsl_multimin_fdfminimizer;
extern const gsl_multimin_fminimizer_type* gsl_multimin_fminimizer_nmsimplex2;
extern const gsl_multimin_fdfminimizer_type* gsl_multimin_fdfminimizer_vector_bfgs2;
gsl_multimin_fminimizer* gsl_multimin_fminimizer_alloc(const gsl_multimin_fminimizer_type* T, size_t n);
int gsl_multimin_fminimizer_set(gsl_multimin_fminimizer* s, gsl_multimin_function* f,
    const gsl_vector* x, const gsl_vector* step_size);
int gsl_multimin_fminimizer_iterate(gsl_multimin_fminimizer* s);
double gsl_multimin_fminimizer_size(const gsl_multimin_fminimizer* s);
void gsl_multimin_fminimizer_free(gsl_multimin_fminimizer* s);
gsl_multimin_fdfminimizer* gsl_multimin_fdfminimizer_alloc(const gsl_multimin_fdfminimizer_type* T, size_t n);
int gsl_multimin_fdfminimizer_set(gsl_multimin_fdfminimizer* s, gsl_multimin_function_fdf* fdf,
    const gsl_vector* x, double step_size, double tol);
int gsl_multimin_fdfminimizer_iterate(gsl_multimin_fdfminimizer* s);
void gsl_multimin_fdfminimizer_free(gsl_multimin_fdfminimizer* s);
int gsl_multimin_test_gradient(const gsl_vector* g, double epsabs);

#ifdef __cplusplus
}
#endif
