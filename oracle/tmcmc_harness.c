/*
 * The reference's TMCMC stage statistics on a given population (test
 * infrastructure: the checker of gliomasolver_b200/tmcmc.py).
 *
 * Compiled with the reference's tools/pi4u_lite/Inference/tmcmc_stats.c
 * (which includes posdef.c) unmodified, against the GSL / MPI / torc
 * stand-ins in oracle/tmcmc_stub (none of the three is installed here; see
 * tmcmc_stub/gsl_stub.h for what the GSL stand-in provides: the simplex search
 * fminsearch reports no convergence, so the reference's own fallback, the grid
 * search fzerofind, sets the next exponent).  This file supplies what the
 * engine's other sources would: the globals data / runinfo / curgen_db
 * (engine_tmcmc.c), the vector helpers compute_max / compute_sum /
 * compute_mean / compute_std with the arithmetic of auxil.c:162-230, the
 * printing helpers, torc_gettime and a multinomial draw that selects nothing
 * (the selection is random and not compared).
 *
 *   tmcmc_harness <population.bin>
 *
 * population.bin: int32 n, int32 d, float64 pj, tolCOV, Tol, then F[n] and
 * the points (n x d, row-major).  Prints one JSON line: the next exponent and
 * the statistics calculate_statistics(F, n, n, 0, sel) leaves in runinfo,
 * fzerofind's own (x, f), and Objlogp at pj + k/8 for k = 1..8.  fzerofind
 * writes fzero_NNN.txt into the working directory.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <sys/time.h>

#include "engine_tmcmc.h"

data_t data;
runinfo_t runinfo;
cgdb_t curgen_db;

double torc_gettime(void)
{
    struct timeval t;
    gettimeofday(&t, NULL);
    return (double)t.tv_sec + (double)t.tv_usec * 1.0E-6;
}

/* auxil.c:162-230 */
double compute_max(double *v, int n)
{
    double m = v[0];
    for (int i = 1; i < n; i++)
        if (v[i] > m) m = v[i];
    return m;
}
double compute_min(double *v, int n)
{
    double m = v[0];
    for (int i = 1; i < n; i++)
        if (v[i] < m) m = v[i];
    return m;
}
double compute_sum(double *v, int n)
{
    double s = 0;
    for (int i = 0; i < n; i++) s += v[i];
    return s;
}
double compute_mean(double *v, int n)
{
    double s = 0;
    for (int i = 0; i < n; i++) s += v[i];
    return s / n;
}
double compute_std(double *v, int n, double mean)
{
    double s = 0;
    for (int i = 0; i < n; i++) s += pow(v[i] - mean, 2);
    return sqrt(s / (n - 1));
}
void print_matrix(char *title, double *v, int n) { (void)title; (void)v; (void)n; }
void print_matrix_2d(char *title, double **v, int n1, int n2) { (void)title; (void)v; (void)n1; (void)n2; }
void multinomialrand(size_t K, unsigned int N, double q[], unsigned int nn[])
{
    (void)N; (void)q;
    for (size_t i = 0; i < K; i++) nn[i] = 0;
}

int fzerofind(double *fj, int fn, double pj, double tol, double *xmin, double *fmin);
void calculate_statistics(double flc[], int n, int nselections, int gen, unsigned int sel[]);
double Objlogp(double x, double *fj, int fn, double pj, double tol);

static void die(const char *m)
{
    fprintf(stderr, "tmcmc_harness: %s\n", m);
    exit(2);
}

int main(int argc, char **argv)
{
    if (argc != 2) die("usage: tmcmc_harness <population.bin>");
    FILE *f = fopen(argv[1], "rb");
    if (!f) die("cannot open input");
    int n = 0, d = 0;
    double hdr[3];
    if (fread(&n, 4, 1, f) != 1 || fread(&d, 4, 1, f) != 1 || n < 2 || d < 1 || fread(hdr, 8, 3, f) != 3)
        die("bad header");
    double *F = malloc(n * sizeof(double)), *pts = malloc((size_t)n * d * sizeof(double));
    if (fread(F, 8, n, f) != (size_t)n || fread(pts, 8, (size_t)n * d, f) != (size_t)n * d) die("short input");
    fclose(f);

    const int G = 4;
    data.Nth = d;
    data.MaxStages = G;
    data.PopSize = n;
    data.TolCOV = hdr[1];
    data.options.MaxIter = 100;
    data.options.Tol = hdr[2];
    data.options.Display = 0;
    data.Num = calloc(G, sizeof(int));
    for (int g = 0; g < G; g++) data.Num[g] = n;
    data.LastNum = n;
    runinfo.CoefVar = calloc(G, sizeof(double));
    runinfo.p = calloc(G, sizeof(double));
    runinfo.currentuniques = calloc(G, sizeof(int));
    runinfo.logselection = calloc(G, sizeof(double));
    runinfo.acceptance = calloc(G, sizeof(double));
    runinfo.SS = malloc(d * sizeof(double *));
    runinfo.SS[0] = calloc((size_t)d * d, sizeof(double)); /* rows contiguous: make_posdef reads SS[0] flat */
    for (int i = 1; i < d; i++) runinfo.SS[i] = runinfo.SS[0] + (size_t)i * d;
    runinfo.meantheta = malloc(G * sizeof(double *));
    for (int g = 0; g < G; g++) runinfo.meantheta[g] = calloc(d, sizeof(double));
    curgen_db.entry = calloc(n, sizeof(cgdbp_t));
    for (int i = 0; i < n; i++) {
        curgen_db.entry[i].point = pts + (size_t)i * d;
        curgen_db.entry[i].F = F[i];
    }
    curgen_db.entries = n;
    runinfo.p[0] = hdr[0];

    double fx = 0, fm = 0;
    const int conv = fzerofind(F, n, hdr[0], hdr[1], &fx, &fm);
    unsigned int *sel = calloc(n, sizeof(unsigned int));
    calculate_statistics(F, n, n, 0, sel);

    printf("{\"p_next\": %.17g, \"coef_var\": %.17g, \"coef_var_next\": %.17g, \"log_selection\": %.17g, "
           "\"fzero\": {\"conv\": %d, \"x\": %.17g, \"f\": %.17g}, \"mean\": [",
           runinfo.p[1], runinfo.CoefVar[0], runinfo.CoefVar[1], runinfo.logselection[0], conv, fx, fm);
    for (int i = 0; i < d; i++) printf("%s%.17g", i ? ", " : "", runinfo.meantheta[0][i]);
    printf("], \"ss\": [");
    for (int i = 0; i < d * d; i++) printf("%s%.17g", i ? ", " : "", runinfo.SS[0][i]);
    printf("], \"objlogp\": [");
    for (int k = 1; k <= 8; k++) printf("%s%.17g", k > 1 ? ", " : "", Objlogp(hdr[0] + k / 8.0, F, n, hdr[0], hdr[1]));
    printf("]}\n");
    return 0;
}
