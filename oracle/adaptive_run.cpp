/*
 * Adaptive forward run (config 2's schedule) on the reference's own MRAG grid,
 * every step and every adaptation by the reference's own code: the oracle of
 * the resident drop-in driver (dropin/glioma_adaptive.cpp).
 *
 * Test infrastructure: compiled with the reference's unmodified sources (see
 * oracle/Makefile, target dropin); no GPU.
 *
 *   adaptive_run <in.bin> <maxlevel> <refine_tol> <compress_tol> <nsteps> <every> ref <out.bin>
 *
 * The grid starts at level 2 (4^3 blocks, periodic, stencil [-1,2)) and is
 * refined with Science::AutomaticRefinement up to <maxlevel>, resampling
 * p_w, p_g, phi from the dense input after every refinement (the fillGrid
 * hook), then compressed once with Science::AutomaticCompression, as the
 * reference's driver does before its time loop
 * (Glioma/Glioma_ReactionDiffusion.cpp:311-313).  Then <nsteps> RD steps,
 * each the reference's pipeline_process + process (:176-187, threaded TBB
 * stand-in); after every <every> steps the grid re-adapts: one loop of
 * Science::AutomaticRefinement (as the driver's in-loop call, :325) and
 * Science::AutomaticCompression to convergence (the driver's commented-out
 * call, :326), interpolation by the reference's own splitter and collapser.
 * Coefficients: Dw = 0.2 cm^2/day on L = 25.6 cm, Dg = Dw/10, rho = 0.05/day,
 * dt = the reference's CFL formula (:304-307) with h of the finest level.
 *
 * Prints one JSON line (blocks and a hash of the sorted (level, index) list
 * after every adaptation; seconds spent stepping and adapting) and writes phi
 * sampled on the finest uniform grid (each finest cell takes the value of the
 * leaf cell that covers it) as int32 n + n^3 float64, x fastest.
 */
#include <sys/time.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "Glioma_Types.h"

static int maxStencil[2][3] = {{-1, -1, -1}, {+2, +2, +2}};

static int g_n = 0;
static std::vector<double> g_pw, g_pg, g_phi;

static void die(const char *m)
{
    fprintf(stderr, "adaptive_run: %s\n", m);
    exit(2);
}

static double now()
{
    timeval tv;
    gettimeofday(&tv, NULL);
    return tv.tv_sec + 1e-6 * tv.tv_usec;
}

static void read_dense(const char *path)
{
    FILE *f = fopen(path, "rb");
    if (!f) die("cannot open input");
    if (fread(&g_n, sizeof(int), 1, f) != 1 || g_n <= 0) die("bad header");
    const size_t N = (size_t)g_n * g_n * g_n;
    g_pw.resize(N);
    g_pg.resize(N);
    g_phi.resize(N);
    if (fread(&g_pw[0], 8, N, f) != N || fread(&g_pg[0], 8, N, f) != N || fread(&g_phi[0], 8, N, f) != N)
        die("short input");
    fclose(f);
}

/* p_w, p_g, phi of every cell sampled from the dense volume at the cell's
 * position, as the reference's _ic maps anatomy voxels
 * (Glioma_ReactionDiffusion.cpp:124-131: floor(x / h_data)). */
static void fill(Grid<W, B> &grid)
{
    std::vector<BlockInfo> vInfo = grid.getBlocksInfo();
    for (size_t i = 0; i < vInfo.size(); i++) {
        const BlockInfo &info = vInfo[i];
        B &block = grid.getBlockCollection()[info.blockID];
        for (int iz = 0; iz < B::sizeZ; iz++)
            for (int iy = 0; iy < B::sizeY; iy++)
                for (int ix = 0; ix < B::sizeX; ix++) {
                    double x[3];
                    info.pos(x, ix, iy, iz);
                    const int gx = (int)floor(x[0] * g_n), gy = (int)floor(x[1] * g_n), gz = (int)floor(x[2] * g_n);
                    const size_t g = (size_t)gx + (size_t)g_n * (gy + (size_t)g_n * gz);
                    block(ix, iy, iz).p_w = (Real)g_pw[g];
                    block(ix, iy, iz).p_g = (Real)g_pg[g];
                    block(ix, iy, iz).phi = (Real)g_phi[g];
                    block(ix, iy, iz).dphidt = 0;
                }
    }
}

/* FNV-1a over the sorted (level, index) list of the leaves */
static unsigned long long leaves_hash(Grid<W, B> &grid, int &nblocks)
{
    std::vector<BlockInfo> vInfo = grid.getBlocksInfo();
    std::vector<std::vector<int> > keys;
    for (size_t i = 0; i < vInfo.size(); i++) {
        std::vector<int> k(4);
        k[0] = vInfo[i].level;
        for (int d = 0; d < 3; d++) k[1 + d] = vInfo[i].index[d];
        keys.push_back(k);
    }
    std::sort(keys.begin(), keys.end());
    unsigned long long h = 1469598103934665603ull;
    for (size_t i = 0; i < keys.size(); i++)
        for (int q = 0; q < 4; q++) {
            const unsigned v = (unsigned)keys[i][q];
            for (int b = 0; b < 4; b++) {
                h ^= (v >> (8 * b)) & 0xffu;
                h *= 1099511628211ull;
            }
        }
    nblocks = (int)keys.size();
    return h;
}

static void ref_step(Grid<W, B> &grid, BlockProcessing &bp, Real Dw, Real Dg, Real rho, double dt)
{
    /* the two calls of Glioma_ReactionDiffusion::_reactionDiffusionStep */
    std::vector<BlockInfo> vInfo = grid.getBlocksInfo();
    const BlockCollection<B> &collecton = grid.getBlockCollection();
    ReactionDiffusionOperator<_DIM> rhs(Dw, Dg, rho);
    UpdateTumor<_DIM> updateTumor(dt);
    bp.pipeline_process(vInfo, collecton, grid.getBoundaryInfo(), rhs);
    BlockProcessing::process(vInfo, collecton, updateTumor, 4);
}

int main(int argc, char **argv)
{
    if (argc != 9)
        die("usage: adaptive_run <in.bin> <maxlevel> <refine_tol> <compress_tol> <nsteps> <every> ref <out.bin>");
    read_dense(argv[1]);
    const int maxLevel = atoi(argv[2]);
    const double rtol = atof(argv[3]), ctol = atof(argv[4]);
    const int nsteps = atoi(argv[5]), every = atoi(argv[6]);
    const std::string mode = argv[7];
    if (g_n != 8 << maxLevel) die("the dense input must have 8 * 2^maxlevel cells per direction");
    if (every <= 0 || nsteps < 0 || mode != "ref") die("bad arguments");

    Refiner_SpaceExtension refiner(1, maxLevel);
    Compressor compressor(1);
    Grid<W, B> grid(4, 4, 4, maxStencil);
    grid.setRefiner(&refiner);
    grid.setCompressor(&compressor);
    fill(grid);
    BlockFWT<W, B, RD_Projector_Wavelets> blockfwt;
    Science::AutomaticRefinement<0, 0>(grid, blockfwt, rtol, maxLevel, -1, NULL, fill);
    Science::AutomaticCompression<0, 0>(grid, blockfwt, ctol, -1, NULL);

    const Real L = (Real)25.6;
    const Real Dw = (Real)((Real)0.2 / (L * L));
    const Real Dg = (Real)(0.1 * Dw);
    const Real rho = (Real)0.05;
    const Real h = (Real)(1. / (8 << maxLevel));
    const Real dt = (Real)(0.99 * h * h / (2. * 3 * (Dw >= Dg ? Dw : Dg)));

    std::vector<int> nblocks;
    std::vector<unsigned long long> hashes;
    int nb0 = 0;
    hashes.push_back(leaves_hash(grid, nb0));
    nblocks.push_back(nb0);

    BlockProcessing ref;
    double t_step = 0, t_adapt = 0;
    long long cell_updates = 0;
    for (int done = 0; done < nsteps;) {
        const int k = std::min(every, nsteps - done);
        const int leaves = (int)grid.getBlocksInfo().size();
        const double t0 = now();
        for (int s = 0; s < k; s++) ref_step(grid, ref, Dw, Dg, rho, dt);
        t_step += now() - t0;
        cell_updates += (long long)k * (long long)leaves * 512;
        done += k;
        const double ta = now();
        Science::AutomaticRefinement<0, 0>(grid, blockfwt, rtol, maxLevel, 1, NULL);
        Science::AutomaticCompression<0, 0>(grid, blockfwt, ctol, -1, NULL);
        t_adapt += now() - ta;
        int nb = 0;
        hashes.push_back(leaves_hash(grid, nb));
        nblocks.push_back(nb);
    }

    /* phi on the finest uniform grid */
    const int n = g_n;
    std::vector<double> out((size_t)n * n * n, 0.0);
    std::vector<BlockInfo> vInfo = grid.getBlocksInfo();
    for (size_t i = 0; i < vInfo.size(); i++) {
        const BlockInfo &info = vInfo[i];
        B &block = grid.getBlockCollection()[info.blockID];
        const int r = 1 << (maxLevel - info.level);
        for (int iz = 0; iz < 8; iz++)
            for (int iy = 0; iy < 8; iy++)
                for (int ix = 0; ix < 8; ix++) {
                    const double v = (double)block(ix, iy, iz).phi;
                    const int x0 = (info.index[0] * 8 + ix) * r, y0 = (info.index[1] * 8 + iy) * r,
                              z0 = (info.index[2] * 8 + iz) * r;
                    for (int dz = 0; dz < r; dz++)
                        for (int dy = 0; dy < r; dy++)
                            for (int dx = 0; dx < r; dx++)
                                out[(size_t)(x0 + dx) + (size_t)n * ((y0 + dy) + (size_t)n * (z0 + dz))] = v;
                }
    }
    FILE *f = fopen(argv[8], "wb");
    if (!f) die("cannot write output");
    fwrite(&n, sizeof(int), 1, f);
    fwrite(&out[0], 8, out.size(), f);
    fclose(f);

    printf("{\"mode\": \"%s\", \"real_bytes\": %d, \"maxlevel\": %d, \"steps\": %d, \"every\": %d, \"dt\": %.17g, "
           "\"step_seconds\": %.6f, \"adapt_seconds\": %.6f, \"cell_updates\": %lld, \"blocks\": [",
           mode.c_str(), (int)sizeof(Real), maxLevel, nsteps, every, (double)dt, t_step, t_adapt, cell_updates);
    for (size_t i = 0; i < nblocks.size(); i++) printf("%s%d", i ? ", " : "", nblocks[i]);
    printf("], \"hashes\": [");
    for (size_t i = 0; i < hashes.size(); i++) printf("%s\"%016llx\"", i ? ", " : "", hashes[i]);
    printf("]}\n");
    return 0;
}
