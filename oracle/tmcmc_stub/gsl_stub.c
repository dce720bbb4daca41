/* The GSL stand-in of gsl_stub.h (test infrastructure; see that header). */
#include "gsl_stub.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static void unreachable(const char *what)
{
    fprintf(stderr, "gsl stand-in: %s is not provided\n", what);
    abort();
}

gsl_vector *gsl_vector_alloc(size_t n)
{
    gsl_vector *v = malloc(sizeof *v);
    v->size = n;
    v->data = calloc(n ? n : 1, sizeof(double));
    return v;
}
void gsl_vector_free(gsl_vector *v)
{
    if (v) { free(v->data); free(v); }
}
double gsl_vector_get(const gsl_vector *v, size_t i) { return v->data[i]; }
void gsl_vector_set(gsl_vector *v, size_t i, double x) { v->data[i] = x; }
void gsl_vector_set_all(gsl_vector *v, double x)
{
    for (size_t i = 0; i < v->size; i++) v->data[i] = x;
}
double gsl_vector_max(const gsl_vector *v)
{
    double m = v->data[0];
    for (size_t i = 1; i < v->size; i++) if (v->data[i] > m) m = v->data[i];
    return m;
}
int gsl_vector_isneg(const gsl_vector *v)
{
    for (size_t i = 0; i < v->size; i++) if (!(v->data[i] < 0)) return 0;
    return 1;
}
int gsl_vector_ispos(const gsl_vector *v)
{
    for (size_t i = 0; i < v->size; i++) if (!(v->data[i] > 0)) return 0;
    return 1;
}

gsl_matrix *gsl_matrix_alloc(size_t n1, size_t n2)
{
    gsl_matrix *m = malloc(sizeof *m);
    m->size1 = n1;
    m->size2 = n2;
    m->data = calloc(n1 * n2 ? n1 * n2 : 1, sizeof(double));
    return m;
}
void gsl_matrix_free(gsl_matrix *m)
{
    if (m) { free(m->data); free(m); }
}
double gsl_matrix_get(const gsl_matrix *m, size_t i, size_t j) { return m->data[i * m->size2 + j]; }
void gsl_matrix_set(gsl_matrix *m, size_t i, size_t j, double x) { m->data[i * m->size2 + j] = x; }
int gsl_matrix_memcpy(gsl_matrix *dst, const gsl_matrix *src)
{
    memcpy(dst->data, src->data, src->size1 * src->size2 * sizeof(double));
    return GSL_SUCCESS;
}
void gsl_matrix_set_identity(gsl_matrix *m)
{
    for (size_t i = 0; i < m->size1; i++)
        for (size_t j = 0; j < m->size2; j++) m->data[i * m->size2 + j] = i == j;
}
int gsl_matrix_fprintf(FILE *f, const gsl_matrix *m, const char *fmt)
{
    for (size_t i = 0; i < m->size1 * m->size2; i++) {
        fprintf(f, fmt, m->data[i]);
        fputc('\n', f);
    }
    return GSL_SUCCESS;
}

gsl_error_handler_t *gsl_set_error_handler_off(void) { return NULL; }

gsl_eigen_symm_workspace *gsl_eigen_symm_alloc(size_t n)
{
    gsl_eigen_symm_workspace *w = malloc(sizeof *w);
    w->n = n;
    return w;
}
void gsl_eigen_symm_free(gsl_eigen_symm_workspace *w) { free(w); }

/* Eigenvalues of a symmetric matrix by cyclic Jacobi rotations (Golub and
 * Van Loan, "Matrix Computations", section 8.5); A is destroyed. */
int gsl_eigen_symm(gsl_matrix *A, gsl_vector *eval, gsl_eigen_symm_workspace *w)
{
    const size_t n = w->n;
    double *a = A->data;
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0;
        for (size_t p = 0; p < n; p++)
            for (size_t q = p + 1; q < n; q++) off += a[p * n + q] * a[p * n + q];
        if (off == 0) break;
        for (size_t p = 0; p < n; p++)
            for (size_t q = p + 1; q < n; q++) {
                const double apq = a[p * n + q];
                if (apq == 0) continue;
                const double theta = (a[q * n + q] - a[p * n + p]) / (2 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1));
                const double c = 1 / sqrt(t * t + 1), s = t * c;
                for (size_t k = 0; k < n; k++) {
                    const double akp = a[k * n + p], akq = a[k * n + q];
                    a[k * n + p] = c * akp - s * akq;
                    a[k * n + q] = s * akp + c * akq;
                }
                for (size_t k = 0; k < n; k++) {
                    const double apk = a[p * n + k], aqk = a[q * n + k];
                    a[p * n + k] = c * apk - s * aqk;
                    a[q * n + k] = s * apk + c * aqk;
                }
            }
    }
    for (size_t i = 0; i < n; i++) eval->data[i] = a[i * n + i];
    return GSL_SUCCESS;
}
gsl_eigen_symmv_workspace *gsl_eigen_symmv_alloc(size_t n)
{
    gsl_eigen_symmv_workspace *w = malloc(sizeof *w);
    w->n = n;
    return w;
}
void gsl_eigen_symmv_free(gsl_eigen_symmv_workspace *w) { free(w); }
int gsl_eigen_symmv(gsl_matrix *A, gsl_vector *e, gsl_matrix *v, gsl_eigen_symmv_workspace *w)
{
    (void)A; (void)e; (void)v; (void)w;
    unreachable("gsl_eigen_symmv");
    return 1;
}
int gsl_blas_dgemm(enum CBLAS_TRANSPOSE ta, enum CBLAS_TRANSPOSE tb, double alpha, const gsl_matrix *A,
                   const gsl_matrix *B, double beta, gsl_matrix *C)
{
    (void)ta; (void)tb; (void)alpha; (void)A; (void)B; (void)beta; (void)C;
    unreachable("gsl_blas_dgemm");
    return 1;
}
int gsl_linalg_cholesky_decomp(gsl_matrix *A) { (void)A; unreachable("gsl_linalg_cholesky_decomp"); return 1; }
int gsl_linalg_cholesky_invert(gsl_matrix *A) { (void)A; unreachable("gsl_linalg_cholesky_invert"); return 1; }

static const gsl_min_fminimizer_type min_type = {0};
const gsl_min_fminimizer_type *gsl_min_fminimizer_brent = &min_type, *gsl_min_fminimizer_goldensection = &min_type,
                              *gsl_min_fminimizer_quad_golden = &min_type;
gsl_min_fminimizer *gsl_min_fminimizer_alloc(const gsl_min_fminimizer_type *T) { (void)T; unreachable("gsl_min"); return NULL; }
void gsl_min_fminimizer_free(gsl_min_fminimizer *s) { (void)s; }
int gsl_min_fminimizer_set(gsl_min_fminimizer *s, gsl_function *f, double x, double lo, double hi)
{ (void)s; (void)f; (void)x; (void)lo; (void)hi; unreachable("gsl_min"); return 1; }
int gsl_min_fminimizer_iterate(gsl_min_fminimizer *s) { (void)s; unreachable("gsl_min"); return 1; }
double gsl_min_fminimizer_x_minimum(const gsl_min_fminimizer *s) { (void)s; unreachable("gsl_min"); return 0; }
double gsl_min_fminimizer_x_lower(const gsl_min_fminimizer *s) { (void)s; unreachable("gsl_min"); return 0; }
double gsl_min_fminimizer_x_upper(const gsl_min_fminimizer *s) { (void)s; unreachable("gsl_min"); return 0; }
double gsl_min_fminimizer_f_minimum(const gsl_min_fminimizer *s) { (void)s; unreachable("gsl_min"); return 0; }
const char *gsl_min_fminimizer_name(const gsl_min_fminimizer *s) { (void)s; return "none"; }
int gsl_min_test_interval(double lo, double hi, double a, double r) { (void)lo; (void)hi; (void)a; (void)r; return 1; }

/* The simplex minimiser reports failure on its first iteration, so that
 * fminsearch returns "not converged". */
static const gsl_multimin_fminimizer_type mm_type = {0};
const gsl_multimin_fminimizer_type *gsl_multimin_fminimizer_nmsimplex = &mm_type,
                                   *gsl_multimin_fminimizer_nmsimplex2 = &mm_type,
                                   *gsl_multimin_fminimizer_nmsimplex2rand = &mm_type;
gsl_multimin_fminimizer *gsl_multimin_fminimizer_alloc(const gsl_multimin_fminimizer_type *T, size_t n)
{
    (void)T;
    gsl_multimin_fminimizer *s = malloc(sizeof *s);
    s->x = gsl_vector_alloc(n);
    s->fval = 0;
    return s;
}
void gsl_multimin_fminimizer_free(gsl_multimin_fminimizer *s)
{
    if (s) { gsl_vector_free(s->x); free(s); }
}
int gsl_multimin_fminimizer_set(gsl_multimin_fminimizer *s, gsl_multimin_function *f, const gsl_vector *x,
                                const gsl_vector *step)
{
    (void)f; (void)step;
    memcpy(s->x->data, x->data, x->size * sizeof(double));
    return GSL_SUCCESS;
}
int gsl_multimin_fminimizer_iterate(gsl_multimin_fminimizer *s) { (void)s; return 1; }
double gsl_multimin_fminimizer_size(const gsl_multimin_fminimizer *s) { (void)s; return 0; }
const char *gsl_multimin_fminimizer_name(const gsl_multimin_fminimizer *s) { (void)s; return "none"; }
int gsl_multimin_test_size(double size, double epsabs) { (void)size; (void)epsabs; return GSL_CONTINUE; }

void gsl_ran_multinomial(const gsl_rng *r, size_t K, unsigned int N, const double p[], unsigned int n[])
{
    (void)r; (void)N; (void)p;
    for (size_t i = 0; i < K; i++) n[i] = 0;
}
double gsl_ran_flat_pdf(double x, double a, double b) { return (x >= a && x < b) ? 1 / (b - a) : 0; }
