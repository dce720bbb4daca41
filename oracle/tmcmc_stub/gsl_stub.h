/*
 * A small stand-in for the parts of the GNU Scientific Library that the
 * reference's TMCMC statistics (tools/pi4u_lite/Inference/tmcmc_stats.c and
 * the posdef.c it includes) name.  GSL is not installed in this image.  Test
 * infrastructure only (oracle/tmcmc_harness.c).
 *
 * Implemented: vectors and matrices (alloc, get/set, copy), the symmetric
 * eigenvalue routine that the positive-definiteness check calls (a Jacobi
 * sweep of our own: only the signs of the eigenvalues are used there), and
 * an error-handler switch.  The simplex minimiser that calculate_statistics
 * tries first (fminsearch, GSL's nmsimplex2) is not restated: its iterate
 * reports failure, so fminsearch returns "not converged" and the reference's
 * own fallback, the grid search fzerofind, sets the next exponent.  Every
 * other routine aborts if reached (none is, for positive definite sample
 * covariances).
 */
#pragma once
#include <float.h> /* GSL's gsl_math.h brings DBL_MAX and the math functions */
#include <math.h>
#include <stddef.h>
#include <stdio.h>

#define GSL_SUCCESS 0
#define GSL_CONTINUE (-2)

typedef struct { size_t size; double *data; } gsl_vector;
typedef struct { size_t size1, size2; double *data; } gsl_matrix;

gsl_vector *gsl_vector_alloc(size_t n);
void gsl_vector_free(gsl_vector *v);
double gsl_vector_get(const gsl_vector *v, size_t i);
void gsl_vector_set(gsl_vector *v, size_t i, double x);
void gsl_vector_set_all(gsl_vector *v, double x);
double gsl_vector_max(const gsl_vector *v);
int gsl_vector_isneg(const gsl_vector *v);
int gsl_vector_ispos(const gsl_vector *v);

gsl_matrix *gsl_matrix_alloc(size_t n1, size_t n2);
void gsl_matrix_free(gsl_matrix *m);
double gsl_matrix_get(const gsl_matrix *m, size_t i, size_t j);
void gsl_matrix_set(gsl_matrix *m, size_t i, size_t j, double x);
int gsl_matrix_memcpy(gsl_matrix *dst, const gsl_matrix *src);
void gsl_matrix_set_identity(gsl_matrix *m);
int gsl_matrix_fprintf(FILE *f, const gsl_matrix *m, const char *fmt);

typedef void gsl_error_handler_t(const char *, const char *, int, int);
gsl_error_handler_t *gsl_set_error_handler_off(void);

typedef struct gsl_eigen_symm_workspace_s { size_t n; } gsl_eigen_symm_workspace;
gsl_eigen_symm_workspace *gsl_eigen_symm_alloc(size_t n);
void gsl_eigen_symm_free(gsl_eigen_symm_workspace *w);
int gsl_eigen_symm(gsl_matrix *A, gsl_vector *eval, gsl_eigen_symm_workspace *w);
typedef struct gsl_eigen_symmv_workspace_s { size_t n; } gsl_eigen_symmv_workspace;
gsl_eigen_symmv_workspace *gsl_eigen_symmv_alloc(size_t n);
void gsl_eigen_symmv_free(gsl_eigen_symmv_workspace *w);
int gsl_eigen_symmv(gsl_matrix *A, gsl_vector *eval, gsl_matrix *evec, gsl_eigen_symmv_workspace *w);

enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112 };
int gsl_blas_dgemm(enum CBLAS_TRANSPOSE ta, enum CBLAS_TRANSPOSE tb, double alpha, const gsl_matrix *A,
                   const gsl_matrix *B, double beta, gsl_matrix *C);
int gsl_linalg_cholesky_decomp(gsl_matrix *A);
int gsl_linalg_cholesky_invert(gsl_matrix *A);

typedef struct { double (*function)(double x, void *params); void *params; } gsl_function;
typedef struct { int dummy; } gsl_min_fminimizer_type;
typedef struct { int dummy; } gsl_min_fminimizer;
extern const gsl_min_fminimizer_type *gsl_min_fminimizer_brent, *gsl_min_fminimizer_goldensection,
    *gsl_min_fminimizer_quad_golden;
gsl_min_fminimizer *gsl_min_fminimizer_alloc(const gsl_min_fminimizer_type *T);
void gsl_min_fminimizer_free(gsl_min_fminimizer *s);
int gsl_min_fminimizer_set(gsl_min_fminimizer *s, gsl_function *f, double x, double lo, double hi);
int gsl_min_fminimizer_iterate(gsl_min_fminimizer *s);
double gsl_min_fminimizer_x_minimum(const gsl_min_fminimizer *s);
double gsl_min_fminimizer_x_lower(const gsl_min_fminimizer *s);
double gsl_min_fminimizer_x_upper(const gsl_min_fminimizer *s);
double gsl_min_fminimizer_f_minimum(const gsl_min_fminimizer *s);
const char *gsl_min_fminimizer_name(const gsl_min_fminimizer *s);
int gsl_min_test_interval(double lo, double hi, double epsabs, double epsrel);

typedef struct {
    double (*f)(const gsl_vector *x, void *params);
    size_t n;
    void *params;
} gsl_multimin_function;
typedef struct { int dummy; } gsl_multimin_fminimizer_type;
typedef struct { gsl_vector *x; double fval; } gsl_multimin_fminimizer;
extern const gsl_multimin_fminimizer_type *gsl_multimin_fminimizer_nmsimplex, *gsl_multimin_fminimizer_nmsimplex2,
    *gsl_multimin_fminimizer_nmsimplex2rand;
gsl_multimin_fminimizer *gsl_multimin_fminimizer_alloc(const gsl_multimin_fminimizer_type *T, size_t n);
void gsl_multimin_fminimizer_free(gsl_multimin_fminimizer *s);
int gsl_multimin_fminimizer_set(gsl_multimin_fminimizer *s, gsl_multimin_function *f, const gsl_vector *x,
                                const gsl_vector *step);
int gsl_multimin_fminimizer_iterate(gsl_multimin_fminimizer *s);
double gsl_multimin_fminimizer_size(const gsl_multimin_fminimizer *s);
const char *gsl_multimin_fminimizer_name(const gsl_multimin_fminimizer *s);
int gsl_multimin_test_size(double size, double epsabs);

typedef struct { int dummy; } gsl_rng;
void gsl_ran_multinomial(const gsl_rng *r, size_t K, unsigned int N, const double p[], unsigned int n[]);
double gsl_ran_flat_pdf(double x, double a, double b);
