/*
 * CPU restatement of GliomaSolver's Fisher-Kolmogorov path (the oracle).
 * TEST INFRASTRUCTURE ONLY -- see rd_oracle.h for who may use it and how it
 * is pinned to the reference.
 *
 * The arithmetic is written with the same operand order and the same
 * Real/double mix as the reference expressions it restates; C's usual
 * arithmetic conversions then round exactly where the C++ reference rounds.
 * Built with -ffp-contract=off so no multiply-add is fused.
 */
#include "rd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define BS 8
#define BS3 512
#define LAB 10 /* lab extent per direction: [-1, 9) */

/* Index of lab position (ix, iy, iz) in [-1,9)^3 among the 488 ghosts, in the
 * order BlockLab::load visits them (MRAGBlockLab.h:256-279); -1 for interior. */
static int g_ghost_id[LAB * LAB * LAB];
static int g_ghost_ready = 0;

static void build_ghost_ids(void)
{
    if (g_ghost_ready) return;
    for (int i = 0; i < LAB * LAB * LAB; i++) g_ghost_id[i] = -1;
    int k = 0;
    for (int icode = 0; icode < 27; icode++) {
        if (icode == 13) continue;
        const int code[3] = {icode % 3 - 1, (icode / 3) % 3 - 1, (icode / 9) % 3 - 1};
        int s[3], e[3];
        for (int d = 0; d < 3; d++) {
            s[d] = code[d] < 1 ? (code[d] < 0 ? -1 : 0) : BS;
            e[d] = code[d] < 1 ? (code[d] < 0 ? 0 : BS) : BS + 1;
        }
        for (int iz = s[2]; iz < e[2]; iz++)
            for (int iy = s[1]; iy < e[1]; iy++)
                for (int ix = s[0]; ix < e[0]; ix++)
                    g_ghost_id[(ix + 1) + LAB * ((iy + 1) + LAB * (iz + 1))] = k++;
    }
    g_ghost_ready = 1;
}

/* ------------------------------------------------------------------------ */
/* ReactionDiffusionOperator<3>::operator() for one cell, given the 7 lab
 * values of (p_w, p_g, phi): index 0 = centre, 1..6 = x-, x+, y-, y+, z-, z+
 * (ReactionDiffusionOperator.h:103-138, _harmonic_mean :148-163,
 * _applyNoFluxBC :166-181). */
#define DEFINE_CELL_RHS(SFX, REAL)                                                      \
    static REAL cell_rhs_##SFX(const REAL *pw, const REAL *pg, const REAL *ph, REAL Dw,  \
                               REAL Dg, REAL rho, double ih2)                            \
    {                                                                                   \
        REAL df[6], chf[6], df_loc;                                                     \
        if (!(pw[0] + pg[0] + ph[0] > 0.)) return (REAL)0.;                             \
        df_loc = pw[0] * Dw + pg[0] * Dg;                                               \
        for (int i = 0; i < 6; i++) df[i] = pw[i + 1] * Dw + pg[i + 1] * Dg;            \
        {                                                                               \
            REAL eps = 1.0e-08;                                                         \
            for (int i = 0; i < 6; i++)                                                 \
                df[i] = (df[i] + df_loc < eps) ? 0. : 2. * df[i] * df_loc / (df[i] + df_loc); \
        }                                                                               \
        for (int i = 0; i < 6; i++) chf[i] = ph[i + 1] + pw[i + 1] + pg[i + 1];         \
        {                                                                               \
            REAL eps = 0.1;                                                             \
            if (chf[0] < eps) { df[1] *= 2.0; }                                         \
            if (chf[1] < eps) { df[0] *= 2.0; }                                         \
            if (chf[2] < eps) { df[3] *= 2.0; }                                         \
            if (chf[3] < eps) { df[2] *= 2.0; }                                         \
            if (chf[4] < eps) { df[5] *= 2.0; }                                         \
            if (chf[5] < eps) { df[4] *= 2.0; }                                         \
        }                                                                               \
        double diffusionFluxIn = ih2 * (df[0] * ph[1] + df[1] * ph[2] + df[2] * ph[3] + \
                                        df[3] * ph[4] + df[4] * ph[5] + df[5] * ph[6]); \
        double diffusionFluxOut =                                                       \
            -((df[0] + df[1] + df[2] + df[3] + df[4] + df[5]) * ph[0] * ih2);            \
        double reactionFlux = rho * ph[0] * (1. - ph[0]);                                \
        return diffusionFluxOut + diffusionFluxIn + reactionFlux;                       \
    }

DEFINE_CELL_RHS(f64, double)
DEFINE_CELL_RHS(f32, float)

/* UpdateTumor<3>::operator() for one cell (ReactionDiffusionOperator.h:
 * 215-222) with MRAG's max/min macros (MRAGCommon.h:19-37). */
#define DEFINE_UPDATE(SFX, REAL)                                                        \
    static inline REAL cell_update_##SFX(REAL phi, REAL dphidt, double dt)             \
    {                                                                                   \
        phi += dt * dphidt;                                                             \
        phi = (((REAL)0.) >= (phi)) ? ((REAL)0.) : (phi);                               \
        phi = (((REAL)1.) < (phi)) ? ((REAL)1.) : (phi);                                \
        return phi;                                                                     \
    }                                                                                   \
    void orc_update_##SFX(int64_t ncells, REAL *phi, const REAL *dphidt, double dt)    \
    {                                                                                   \
        for (int64_t i = 0; i < ncells; i++) phi[i] = cell_update_##SFX(phi[i], dphidt[i], dt); \
    }

DEFINE_UPDATE(f64, double)
DEFINE_UPDATE(f32, float)

/* ------------------------------------------------------------------------ */
/* Dense periodic grid. */
#define DEFINE_DENSE(SFX, REAL)                                                         \
    void orc_rd_rhs_dense_##SFX(int n, const REAL *pw, const REAL *pg, const REAL *phi,  \
                                REAL Dw, REAL Dg, REAL rho, REAL hr, REAL *dphidt)       \
    {                                                                                   \
        double h = hr;                                                                  \
        double ih2 = 1. / (h * h);                                                      \
        const int64_t nn = n;                                                           \
        for (int iz = 0; iz < n; iz++)                                                  \
            for (int iy = 0; iy < n; iy++)                                              \
                for (int ix = 0; ix < n; ix++) {                                        \
                    const int xm = (ix + n - 1) % n, xp = (ix + 1) % n;                 \
                    const int ym = (iy + n - 1) % n, yp = (iy + 1) % n;                 \
                    const int zm = (iz + n - 1) % n, zp = (iz + 1) % n;                 \
                    const int64_t id[7] = {                                             \
                        ix + nn * (iy + nn * iz), xm + nn * (iy + nn * iz),             \
                        xp + nn * (iy + nn * iz), ix + nn * (ym + nn * iz),             \
                        ix + nn * (yp + nn * iz), ix + nn * (iy + nn * zm),             \
                        ix + nn * (iy + nn * zp)};                                      \
                    REAL a[7], b[7], c[7];                                              \
                    for (int k = 0; k < 7; k++) {                                       \
                        a[k] = pw[id[k]]; b[k] = pg[id[k]]; c[k] = phi[id[k]];          \
                    }                                                                   \
                    dphidt[id[0]] = cell_rhs_##SFX(a, b, c, Dw, Dg, rho, ih2);          \
                }                                                                       \
    }

DEFINE_DENSE(f64, double)
DEFINE_DENSE(f32, float)

void orc_rd_steps_dense_f64(int n, const double *pw, const double *pg, double *phi,
                            double Dw, double Dg, double rho, double h, double dt, int nsteps,
                            double *scratch)
{
    const int64_t N = (int64_t)n * n * n;
    for (int s = 0; s < nsteps; s++) {
        orc_rd_rhs_dense_f64(n, pw, pg, phi, Dw, Dg, rho, h, scratch);
        orc_update_f64(N, phi, scratch, dt);
    }
}

void orc_rd_steps_dense_f32(int n, const float *pw, const float *pg, float *phi,
                            float Dw, float Dg, float rho, float h, double dt, int nsteps,
                            float *scratch)
{
    const int64_t N = (int64_t)n * n * n;
    for (int s = 0; s < nsteps; s++) {
        orc_rd_rhs_dense_f32(n, pw, pg, phi, Dw, Dg, rho, h, scratch);
        orc_update_f32(N, phi, scratch, dt);
    }
}

/* ------------------------------------------------------------------------ */
/* Block pool with lab ghosts. */
#define DEFINE_POOL(SFX, REAL)                                                          \
    void orc_fill_ghosts_##SFX(const orc_ghost_csr *g, const REAL *field, REAL *out)    \
    {                                                                                   \
        for (int64_t r = 0; r < g->nrows; r++) {                                        \
            REAL ghost = 0;                                                             \
            for (int64_t k = g->row_ptr[r]; k < g->row_ptr[r + 1]; k++) {               \
                const REAL w = ((REAL)g->w0[k] * (REAL)g->w1[k]) * (REAL)g->w2[k];      \
                ghost += field[g->src[k]] * w;                                          \
            }                                                                           \
            out[r] = ghost;                                                             \
        }                                                                               \
    }                                                                                   \
    static inline REAL lab_##SFX(const REAL *blk, const REAL *ghosts, int ix, int iy, int iz) \
    {                                                                                   \
        if (ix >= 0 && ix < BS && iy >= 0 && iy < BS && iz >= 0 && iz < BS)             \
            return blk[ix + BS * (iy + BS * iz)];                                       \
        return ghosts[g_ghost_id[(ix + 1) + LAB * ((iy + 1) + LAB * (iz + 1))]];        \
    }                                                                                   \
    void orc_rd_rhs_pool_##SFX(int nblocks, const REAL *h, const REAL *pw, const REAL *pg, \
                               const REAL *phi, const REAL *gpw, const REAL *gpg,        \
                               const REAL *gphi, REAL Dw, REAL Dg, REAL rho, REAL *dphidt) \
    {                                                                                   \
        build_ghost_ids();                                                              \
        static const int off[7][3] = {{0, 0, 0}, {-1, 0, 0}, {1, 0, 0}, {0, -1, 0},     \
                                      {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};                \
        for (int b = 0; b < nblocks; b++) {                                             \
            double hb = h[b];                                                           \
            double ih2 = 1. / (hb * hb);                                                \
            const REAL *bw = pw + (int64_t)b * BS3, *bg = pg + (int64_t)b * BS3;        \
            const REAL *bp = phi + (int64_t)b * BS3;                                    \
            const REAL *gw = gpw + (int64_t)b * ORC_LAB_GHOSTS;                         \
            const REAL *gg = gpg + (int64_t)b * ORC_LAB_GHOSTS;                         \
            const REAL *gp = gphi + (int64_t)b * ORC_LAB_GHOSTS;                        \
            for (int iz = 0; iz < BS; iz++)                                             \
                for (int iy = 0; iy < BS; iy++)                                         \
                    for (int ix = 0; ix < BS; ix++) {                                   \
                        REAL a[7], bb[7], c[7];                                         \
                        for (int k = 0; k < 7; k++) {                                   \
                            const int x = ix + off[k][0], y = iy + off[k][1], z = iz + off[k][2]; \
                            a[k] = lab_##SFX(bw, gw, x, y, z);                          \
                            bb[k] = lab_##SFX(bg, gg, x, y, z);                         \
                            c[k] = lab_##SFX(bp, gp, x, y, z);                          \
                        }                                                               \
                        dphidt[(int64_t)b * BS3 + ix + BS * (iy + BS * iz)] =           \
                            cell_rhs_##SFX(a, bb, c, Dw, Dg, rho, ih2);                 \
                    }                                                                   \
        }                                                                               \
    }

DEFINE_POOL(f64, double)
DEFINE_POOL(f32, float)

/* ------------------------------------------------------------------------ */
/* Interpolating 2nd-order wavelets (MRAG/MRAGcore/MRAGWavelets_StaticData.cpp:
 * 13-21): Ha = {1} on [0,1), Ga = {-.5, 1, -.5} on [-2,1), Hs = {.5, 1, .5}
 * on [-1,2). */
static const double kGa[3] = {-0.5, 1., -0.5};
static const double kHs[3] = {0.5, 1., 0.5};

/* BlockFWT::_filter (MRAGBlockFWT.h:219-257): for subband bits (wx, wy, wz) the
 * filter runs z, then y, then x over the support, reading lab(o - i), and
 * accumulates phi * (wZ*wY * wX) in Real. */
#define DEFINE_FWT(SFX, REAL)                                                           \
    static REAL fwt_filter_##SFX(const REAL *blk, const REAL *gh, int wx, int wy, int wz, \
                                 int dx, int dy, int dz)                                 \
    {                                                                                   \
        const REAL Ga[3] = {(REAL)kGa[0], (REAL)kGa[1], (REAL)kGa[2]};                  \
        const REAL Ha0 = (REAL)1;                                                       \
        const int s[3] = {wx ? -2 : 0, wy ? -2 : 0, wz ? -2 : 0};                       \
        const int e[3] = {1, 1, 1};                                                     \
        const int o[3] = {2 * dx, 2 * dy, 2 * dz};                                      \
        REAL result = 0;                                                                \
        for (int iz = s[2]; iz < e[2]; iz++) {                                          \
            const REAL wZ = wz ? Ga[iz + 2] : Ha0;                                      \
            for (int iy = s[1]; iy < e[1]; iy++) {                                      \
                const REAL wY = wy ? Ga[iy + 2] : Ha0;                                  \
                const REAL wZwY = wZ * wY;                                              \
                for (int ix = s[0]; ix < e[0]; ix++) {                                  \
                    const REAL wX = wx ? Ga[ix + 2] : Ha0;                              \
                    result += lab_##SFX(blk, gh, o[0] - ix, o[1] - iy, o[2] - iz) * (wZwY * wX); \
                }                                                                       \
            }                                                                           \
        }                                                                               \
        return result;                                                                  \
    }                                                                                   \
    void orc_fwt_detail_pool_##SFX(int nblocks, const REAL *phi, const REAL *gphi, double *out) \
    {                                                                                   \
        build_ghost_ids();                                                              \
        for (int b = 0; b < nblocks; b++) {                                             \
            const REAL *blk = phi + (int64_t)b * BS3;                                   \
            const REAL *gh = gphi + (int64_t)b * ORC_LAB_GHOSTS;                        \
            double maxv[8] = {0, 0, 0, 0, 0, 0, 0, 0};                                  \
            for (int iz = 0; iz < BS / 2; iz++)                                         \
                for (int iy = 0; iy < BS / 2; iy++)                                     \
                    for (int ix = 0; ix < BS / 2; ix++)                                 \
                        for (int code = 0; code < 8; code++) {                          \
                            const REAL v = fwt_filter_##SFX(blk, gh, code & 1, (code >> 1) & 1, \
                                                            (code >> 2) & 1, ix, iy, iz); \
                            const double a = fabs(v);                                   \
                            if (!(a < maxv[code])) maxv[code] = a;                      \
                        }                                                               \
            double m = maxv[1];                                                         \
            for (int code = 2; code < 8; code++) m = (m < maxv[code]) ? maxv[code] : m; \
            out[b] = m;                                                                 \
        }                                                                               \
    }

DEFINE_FWT(f64, double)
DEFINE_FWT(f32, float)

/* BlockSplitter::_splitBlocks (MRAGBlockSplitter.h:49-98) for Interp2ndOrder:
 * coarse lab points s in [0, 9)^3 (z, y, x order) scatter to fine points d in
 * [2s-1, 2s+2) clipped to [0,16) with weight Hs(2s-d), the weight product in
 * double (wZ*wY)*wX and then converted to Real (Cell*Real, Glioma_Types.h). */
#define DEFINE_SPLIT(SFX, REAL)                                                         \
    void orc_split_block_##SFX(const REAL *parent, const REAL *gparent, REAL *children) \
    {                                                                                   \
        build_ghost_ids();                                                              \
        memset(children, 0, sizeof(REAL) * 8 * BS3);                                    \
        for (int sz = 0; sz < BS + 1; sz++)                                             \
            for (int sy = 0; sy < BS + 1; sy++)                                         \
                for (int sx = 0; sx < BS + 1; sx++) {                                   \
                    const int st[3] = {2 * sx - 1 < 0 ? 0 : 2 * sx - 1,                 \
                                       2 * sy - 1 < 0 ? 0 : 2 * sy - 1,                 \
                                       2 * sz - 1 < 0 ? 0 : 2 * sz - 1};                \
                    const int en[3] = {2 * sx + 2 > 2 * BS ? 2 * BS : 2 * sx + 2,        \
                                       2 * sy + 2 > 2 * BS ? 2 * BS : 2 * sy + 2,        \
                                       2 * sz + 2 > 2 * BS ? 2 * BS : 2 * sz + 2};       \
                    const REAL v = lab_##SFX(parent, gparent, sx, sy, sz);              \
                    for (int dz = st[2]; dz < en[2]; dz++) {                            \
                        const double wZ = kHs[2 * sz - dz + 1];                         \
                        for (int dy = st[1]; dy < en[1]; dy++) {                        \
                            const double wY = kHs[2 * sy - dy + 1];                     \
                            const double wZwY = wZ * wY;                                \
                            for (int dx = st[0]; dx < en[0]; dx++) {                    \
                                const int cx = dx / BS, cy = dy / BS, cz = dz / BS;     \
                                REAL *child = children + (cx + 2 * (cy + 2 * cz)) * BS3; \
                                const REAL w = (REAL)(wZwY * kHs[2 * sx - dx + 1]);     \
                                child[(dx - cx * BS) + BS * ((dy - cy * BS) + BS * (dz - cz * BS))] += v * w; \
                            }                                                           \
                        }                                                               \
                    }                                                                   \
                }                                                                       \
    }                                                                                   \
    void orc_collapse_blocks_##SFX(const REAL *children, REAL *parent)                  \
    {                                                                                   \
        for (int c = 0; c < 8; c++) {                                                   \
            const int cx = c & 1, cy = (c >> 1) & 1, cz = (c >> 2) & 1;                 \
            const REAL *src = children + c * BS3;                                       \
            for (int iz = 0; iz < BS / 2; iz++)                                         \
                for (int iy = 0; iy < BS / 2; iy++)                                     \
                    for (int ix = 0; ix < BS / 2; ix++) {                               \
                        REAL r = 0;                                                     \
                        r += src[2 * ix + BS * (2 * iy + BS * 2 * iz)] * (REAL)(1.0 * 1.0 * 1.0); \
                        parent[(cx * 4 + ix) + BS * ((cy * 4 + iy) + BS * (cz * 4 + iz))] = r; \
                    }                                                                   \
        }                                                                               \
    }

DEFINE_SPLIT(f64, double)
DEFINE_SPLIT(f32, float)

/* ------------------------------------------------------------------------ */
/* _dumpUQoutput (Glioma_ReactionDiffusion.cpp:208-262). */
#define DEFINE_UQ_DUMP(SFX, REAL)                                                       \
    void orc_uq_dump_##SFX(int nblocks, const int *level, const int *index, const REAL *h, \
                           const REAL *phi, int gpd, double *out)                        \
    {                                                                                   \
        const double hf = 1. / gpd;                                                     \
        const double eps = hf * 0.5;                                                    \
        memset(out, 0, sizeof(double) * (size_t)gpd * gpd * gpd);                       \
        for (int b = 0; b < nblocks; b++) {                                             \
            const double dilate = ldexp(1.0, -level[b]);                                \
            const REAL origin[3] = {(REAL)(index[3 * b] * dilate), (REAL)(index[3 * b + 1] * dilate), \
                                    (REAL)(index[3 * b + 2] * dilate)};                 \
            const REAL hb = h[b];                                                       \
            const double hd = hb;                                                       \
            for (int iz = 0; iz < BS; iz++)                                             \
                for (int iy = 0; iy < BS; iy++)                                         \
                    for (int ix = 0; ix < BS; ix++) {                                   \
                        const double x0 = origin[0] + hb * ix;                          \
                        const double x1 = origin[1] + hb * iy;                          \
                        const double x2 = origin[2] + hb * iz;                          \
                        const int mx = (int)floor(x0 / hf), my = (int)floor(x1 / hf),   \
                                  mz = (int)floor(x2 / hf);                              \
                        const double v = phi[(int64_t)b * BS3 + ix + BS * (iy + BS * iz)]; \
                        int c;                                                          \
                        if (hd < hf + eps) c = 1;                                       \
                        else if (hd < 2. * hf + eps) c = 2;                             \
                        else if (hd < 3. * hf + eps) c = 3;                             \
                        else c = 4;                                                     \
                        for (int cz = 0; cz < c; cz++)                                  \
                            for (int cy = 0; cy < c; cy++)                              \
                                for (int cx = 0; cx < c; cx++)                          \
                                    out[(mx + cx) + (size_t)gpd * ((my + cy) + (size_t)gpd * (mz + cz))] = v; \
                    }                                                                   \
        }                                                                               \
    }

DEFINE_UQ_DUMP(f64, double)
DEFINE_UQ_DUMP(f32, float)

/* HGG_Likelihood::_computeLogBernoulli (HGG_Likelihood.cpp:136-163). */
static long double log_bernoulli(double u, double y, double uc, double slope)
{
    const double is2 = 1. / slope;
    const double diff = u - uc;
    const long double omega2 = (diff > 0.) ? 1. : diff * diff;
    const int sgn = (diff < -0.0) ? -1 : (diff > 0.0);
    const long double alpha = 0.5 + 0.5 * sgn * (1. - expl(-omega2 * is2));
    return (y == 1) ? logl(alpha) : logl(1. - alpha);
}

void orc_log_likelihood(int n, const double *model, const double *t1c, const double *flair, const double *pet,
                        const int *roi, int nroi, double pet_sigma2, double pet_scale, double t1uc,
                        double t2uc, double slope, int step_pet, int step_mri, long double out[3])
{
    /* PET (HGG_Likelihood.cpp:40-75) */
    out[0] = 0;
    if (pet) {
        int N = 0;
        long double sum = 0.;
        for (int iz = 0; iz < n; iz++)
            for (int iy = 0; iy < n; iy++)
                for (int ix = 0; ix < n; ix++) {
                    if ((ix % step_pet == 0) && (iy % step_pet == 0) && (iz % step_pet == 0)) {
                        const size_t g = ix + (size_t)n * (iy + (size_t)n * iz);
                        if (pet[g] > 0.) {
                            sum += (model[g] - pet_scale * pet[g]) * (model[g] - pet_scale * pet[g]);
                            N++;
                        }
                    }
                }
        const long double p1 = -0.5 * N * log(2. * M_PI * pet_sigma2);
        const long double p2 = -0.5 * (1. / pet_sigma2) * sum;
        out[0] = p1 + p2;
    }
    /* T1c, FLAIR (:77-128) */
    for (int ti = 1; ti <= 2; ti++) {
        const double *data = ti == 1 ? t1c : flair;
        const double uc = ti == 1 ? t1uc : t2uc;
        long double sum = 0.;
        if (!roi) {
            for (size_t g = 0; g < (size_t)n * n * n; g++) sum += log_bernoulli(model[g], data[g], uc, slope);
        } else {
            for (int i = 0; i < nroi; i++) {
                const int ix = roi[3 * i], iy = roi[3 * i + 1], iz = roi[3 * i + 2];
                if ((ix % step_mri == 0) && (iy % step_mri == 0) && (iz % step_mri == 0)) {
                    const size_t g = ix + (size_t)n * (iy + (size_t)n * iz);
                    sum += log_bernoulli(model[g], data[g], uc, slope);
                }
            }
        }
        out[ti] = sum;
    }
}

/* Glioma_ReactionDiffusion::_ic (Glioma/Glioma_ReactionDiffusion.cpp:79-172),
 * restated cell by cell in the build's Real.  In the float build the
 * reference mixes float and double: the voxel index divides a float
 * position by a double spacing (:125-127), `double tissue = pWM + pGM` adds
 * in float (:144,149), the normalisation divides in double (:150-151), the
 * tumour distance is float (:155-157) and the smoothing profile evaluates
 * (1 - psi) in float and the rest in double (:161-162). */
#define ORC_MAP_ANATOMY(SUF, Real, SQRT)                                                                        \
    void orc_map_anatomy_##SUF(int bpd, int sx, int sy, int sz, const double *gm, const double *wm,             \
                               const double *csf, const double tumor_ic[3], Real *pw, Real *pg, Real *pcsf,     \
                               Real *phi, Real *tissue_out)                                                     \
    {                                                                                                          \
        int level = 0;                                                                                         \
        while ((1 << level) < bpd) level++;                                                                    \
        const int n = 8 * bpd;                                                                                 \
        const Real hcell = (Real)(1.0 / (8 << level)); /* BlockInfo::h = 2^-level / 8 */                       \
        int smax = sx > sy ? sx : sy;                                                                          \
        smax = smax > sz ? smax : sz;                                                                          \
        const double brainHx = 1.0 / ((double)smax); /* :98 */                                                 \
        const Real tumorRadius = 0.005, smooth_sup = 2., hs = 1. / 128; /* :103-105 */                         \
        const Real iw = 1. / (smooth_sup * hs);                           /* :106 */                           \
        const Real ic[3] = {(Real)tumor_ic[0], (Real)tumor_ic[1], (Real)tumor_ic[2]};                          \
        for (int iz = 0; iz < n; iz++)                                                                         \
            for (int iy = 0; iy < n; iy++)                                                                     \
                for (int ix = 0; ix < n; ix++) {                                                               \
                    const size_t c = ix + (size_t)n * (iy + (size_t)n * iz);                                   \
                    /* origin = (i / 8) * 8 * hcell, + hcell * (i % 8): exact either way */                    \
                    Real x[3];                                                                                 \
                    x[0] = (Real)((ix / 8) * 8) * hcell + hcell * (ix % 8);                                    \
                    x[1] = (Real)((iy / 8) * 8) * hcell + hcell * (iy % 8);                                    \
                    x[2] = (Real)((iz / 8) * 8) * hcell + hcell * (iz % 8);                                    \
                    const int mX = (int)floor(x[0] / brainHx);                                                 \
                    const int mY = (int)floor(x[1] / brainHx);                                                 \
                    const int mZ = (int)floor(x[2] / brainHx);                                                 \
                    Real o_w = 0, o_g = 0, o_c = 0, o_phi = 0, o_t = 0;                                        \
                    if (mX >= 0 && mX < sx && mY >= 0 && mY < sy && mZ >= 0 && mZ < sz) {                      \
                        const size_t v = mX + (size_t)sx * (mY + (size_t)sy * mZ);                             \
                        Real pGM = gm[v], pWM = wm[v], pCSF = csf[v];                                          \
                        double tissue = pWM + pGM;                                                             \
                        pCSF = (pCSF > tissue) ? 1. : 0.;                                                      \
                        pWM = (pCSF > tissue) ? 0. : pWM;                                                      \
                        pGM = (pCSF > tissue) ? 0. : pGM;                                                      \
                        tissue = pWM + pGM;                                                                    \
                        o_w = (tissue > 0.) ? (pWM / tissue) : 0.;                                             \
                        o_g = (tissue > 0.) ? (pGM / tissue) : 0.;                                             \
                        o_c = pCSF;                                                                            \
                        o_t = pGM + pWM;                                                                       \
                        const Real p[3] = {x[0] - ic[0], x[1] - ic[1], x[2] - ic[2]};                          \
                        const Real dist = SQRT(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);                       \
                        const Real psi = (dist - tumorRadius) * iw;                                            \
                        if ((psi < -1) && (pGM + pWM > 0.001))                                                 \
                            o_phi = 1.0;                                                                       \
                        else if (((-1 <= psi) && (psi <= 1)) && (pGM + pWM > 0))                               \
                            o_phi = 1.0 * 0.5 * (1 - psi - sin(M_PI * psi) / (M_PI));                          \
                        else                                                                                   \
                            o_phi = 0.0;                                                                       \
                    }                                                                                          \
                    if (pw) pw[c] = o_w;                                                                       \
                    if (pg) pg[c] = o_g;                                                                       \
                    if (pcsf) pcsf[c] = o_c;                                                                   \
                    if (phi) phi[c] = o_phi;                                                                   \
                    if (tissue_out) tissue_out[c] = o_t;                                                       \
                }                                                                                              \
    }
ORC_MAP_ANATOMY(f64, double, sqrt)
ORC_MAP_ANATOMY(f32, float, sqrtf)

/* ------------------------------------------------------------------------ */
/* The discrete adjoint of one fused step on a dense periodic grid, FP64: the
 * derivative of the step of orc_rd_steps_dense_f64 (ReactionDiffusionOperator
 * + UpdateTumor, ReactionDiffusionOperator.h:97-138,189-226) with its
 * piecewise-constant switches held fixed: the domain test, the no-flux
 * doubling of the coefficient opposite a neighbour with chf < 0.1, the clamp
 * (derivative 1 where 0 < phi + dt*dphidt <= 1).  With
 *   r_i = ih2 sum_k df_ik phi_k - ih2 (sum_k df_ik) phi_i + rho phi_i (1 - phi_i)
 * (df_ik the doubled harmonic mean towards neighbour k, 0 outside the domain):
 *   mu_i     = lam'_i [0 < pre_i <= 1]
 *   lam_j    = mu_j + dt ( dom_j mu_j (-ih2 sum_k df_jk + rho (1 - 2 phi_j))
 *                         + ih2 sum_{k} dom_i mu_i df_i,k^1 ),  i = j + e_k
 *   grad[0] += sum_i dom_i mu_i dt phi_i (1 - phi_i)             (d / d rho)
 *   grad[1] += sum_i dom_i mu_i dt (diffusive part of r_i) / Dw   (d / d Dw, Dg = 0.1 Dw:
 *              the coefficients are homogeneous of degree 1 in Dw)
 * phi is the state the step maps forward; lam holds dL/dphi' on entry and
 * dL/dphi on exit; scratch holds 8 n^3 doubles. */
void orc_adjoint_step_dense_f64(int n, const double *pw, const double *pg, const double *phi, double Dw,
                                double Dg, double rho, double h, double dt, double *lam, double grad[4],
                                double *scratch)
{
    const int64_t nn = n, N = nn * nn * nn;
    const double ih2 = 1. / (h * h);
    double *mu = scratch, *dom = scratch + N, *dfs = scratch + 2 * N; /* dfs: 6 per cell */
    for (int iz = 0; iz < n; iz++)
        for (int iy = 0; iy < n; iy++)
            for (int ix = 0; ix < n; ix++) {
                const int xm = (ix + n - 1) % n, xp = (ix + 1) % n;
                const int ym = (iy + n - 1) % n, yp = (iy + 1) % n;
                const int zm = (iz + n - 1) % n, zp = (iz + 1) % n;
                const int64_t id[7] = {ix + nn * (iy + nn * iz), xm + nn * (iy + nn * iz), xp + nn * (iy + nn * iz),
                                       ix + nn * (ym + nn * iz), ix + nn * (yp + nn * iz), ix + nn * (iy + nn * zm),
                                       ix + nn * (iy + nn * zp)};
                const int64_t c = id[0];
                double a[7], b[7], p[7], df[6] = {0, 0, 0, 0, 0, 0};
                for (int k = 0; k < 7; k++) {
                    a[k] = pw[id[k]];
                    b[k] = pg[id[k]];
                    p[k] = phi[id[k]];
                }
                const int d = a[0] + b[0] + p[0] > 0.;
                double dphidt = 0., diff = 0.;
                if (d) {
                    const double df_loc = a[0] * Dw + b[0] * Dg;
                    for (int k = 0; k < 6; k++) {
                        const double dn = a[k + 1] * Dw + b[k + 1] * Dg;
                        df[k] = (dn + df_loc < 1.0e-08) ? 0. : 2. * dn * df_loc / (dn + df_loc);
                    }
                    for (int k = 0; k < 6; k++)
                        if (p[k + 1] + a[k + 1] + b[k + 1] < 0.1) df[k ^ 1] *= 2.0;
                    const double in = ih2 * (df[0] * p[1] + df[1] * p[2] + df[2] * p[3] + df[3] * p[4] +
                                             df[4] * p[5] + df[5] * p[6]);
                    const double out = -((df[0] + df[1] + df[2] + df[3] + df[4] + df[5]) * p[0] * ih2);
                    dphidt = out + in + rho * p[0] * (1. - p[0]);
                    diff = out + in;
                }
                const double pre = p[0] + dt * dphidt;
                const int pass = pre > 0. && pre <= 1.;
                mu[c] = pass ? lam[c] : 0.;
                dom[c] = d;
                for (int k = 0; k < 6; k++) dfs[6 * c + k] = df[k];
                if (d && pass) {
                    const double tr = mu[c] * dt * p[0] * (1. - p[0]), td = mu[c] * dt * diff / Dw;
                    grad[0] += tr;
                    grad[1] += td;
                    grad[2] += fabs(tr);
                    grad[3] += fabs(td);
                }
            }
    for (int iz = 0; iz < n; iz++)
        for (int iy = 0; iy < n; iy++)
            for (int ix = 0; ix < n; ix++) {
                const int xm = (ix + n - 1) % n, xp = (ix + 1) % n;
                const int ym = (iy + n - 1) % n, yp = (iy + 1) % n;
                const int zm = (iz + n - 1) % n, zp = (iz + 1) % n;
                const int64_t c = ix + nn * (iy + nn * iz);
                const int64_t nb[6] = {xm + nn * (iy + nn * iz), xp + nn * (iy + nn * iz), ix + nn * (ym + nn * iz),
                                       ix + nn * (yp + nn * iz), ix + nn * (iy + nn * zm), ix + nn * (iy + nn * zp)};
                double acc = 0.;
                if (dom[c]) {
                    double sdf = 0.;
                    for (int k = 0; k < 6; k++) sdf += dfs[6 * c + k];
                    acc += mu[c] * (-ih2 * sdf + rho * (1. - 2. * phi[c]));
                }
                for (int k = 0; k < 6; k++)
                    if (dom[nb[k]]) acc += ih2 * dfs[6 * nb[k] + (k ^ 1)] * mu[nb[k]];
                lam[c] = mu[c] + dt * acc;
            }
}

/* d loss / du of loss = -(L_T1c + L_FLAIR) (HGG_Likelihood.cpp:136-156): the
 * Bernoulli term with alpha = 1/2 + 1/2 sgn(u - uc) (1 - exp(-w2 / slope)),
 * w2 = 1 above uc and (u - uc)^2 below, differentiated: above uc the terms are
 * constant; below, with d = u - uc and e = exp(-d^2 / slope),
 * d log(alpha) / du = -2 d / slope and d log(1 - alpha) / du = e d / slope / (1 - e/2). */
void orc_loss_grad_f64(int64_t ncells, const double *u, const double *t1c, const double *flair, double t1uc,
                       double t2uc, double slope, double *lam)
{
    for (int64_t i = 0; i < ncells; i++) {
        double g = 0.;
        for (int t = 0; t < 2; t++) {
            const double d = u[i] - (t ? t2uc : t1uc);
            const int y = (t ? flair[i] : t1c[i]) == 1.;
            if (!(d < -0.0)) continue;
            const double e = exp(-d * d / slope);
            g += y ? -2. * d / slope : e * d / slope / (1. - 0.5 * e);
        }
        lam[i] = -g;
    }
}
