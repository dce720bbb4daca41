/*
 * glioma_adaptive: the adaptive Fisher-Kolmogorov forward run with its leaves
 * resident on the GPU from the first step to the last.
 *
 * This is the reference's driver loop (Glioma/Glioma_ReactionDiffusion.cpp:
 * 300-334) with the drop-in: the block tree is the reference's own MRAG grid
 * (compiled from its sources), every RD step is one gbfk_rd_step launch
 * (plus a ghost fill of coarse-fine faces), and each re-adaptation runs
 * gbfk_mrag::AutomaticRefinement / AutomaticCompression: wavelet details on
 * the device, the grid's own refine/compress plans, split and collapse on the
 * device through the grid's splitter and collapser hooks
 * (include/gbfk_mrag.hpp).  phi is uploaded once and read back once, at the
 * end.
 *
 *   glioma_adaptive <in.bin> <maxlevel> <refine_tol> <compress_tol> <nsteps> <every> <out.bin>
 *                   [<Dw cm^2/day> <rho /day>]
 *
 * in.bin: int32 n, then p_w, p_g, phi as n^3 float64 each, x fastest,
 * n = 8 * 2^maxlevel.  The grid starts at level 2 (4^3 blocks, periodic,
 * stencil [-1,2)) and is refined on the host with the reference's
 * Science::AutomaticRefinement up to <maxlevel>, resampling the fields from
 * the dense input after every refinement, then compressed once with
 * Science::AutomaticCompression (the driver's set-up before its time loop,
 * :311-313); the leaves then move to the GPU.  Then <nsteps> RD steps; after
 * every <every> steps one loop of refinement (the driver's in-loop call,
 * :325) and compression to convergence (its commented-out call, :326);
 * <every> = 0 keeps the set-up's grid for the whole run.
 * Coefficients: Dw = 0.2 cm^2/day (or the optional argument) on L = 25.6 cm,
 * Dg = Dw/10, rho = 0.05/day (or the optional argument), dt = the
 * reference's CFL formula (:304-307) with h of the finest level (the
 * driver's h of the initial grid is unstable once blocks reach level 5).
 *
 * Prints one JSON line: blocks and an FNV-1a hash of the sorted
 * (level, index) leaf list after every adaptation; seconds of device stepping,
 * of the adaptation and of its parts; the decisions whose detail lay within
 * 1e-6 (relative) of its tolerance.  Writes phi sampled on the finest uniform
 * grid as int32 n + n^3 float64, x fastest (each leaf cell's value on the r^3
 * finest cells it covers, r = 2^(maxlevel - level), its own position
 * origin + h * index being the first of them), and the leaves' levels on
 * the same grid to <out.bin>.levels (n^3 int8).
 */
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "Glioma_Types.h"
#include "gbfk_mrag.hpp"

typedef Grid<W, B> GridT;

static int maxStencil[2][3] = {{-1, -1, -1}, {+2, +2, +2}};
static int g_n = 0;
static std::vector<double> g_pw, g_pg, g_phi;

/* %.6e, or null for a value JSON cannot hold (a margin no decision set) */
static std::string json_number(double v)
{
    if (!std::isfinite(v)) return "null";
    char b[32];
    snprintf(b, sizeof b, "%.6e", v);
    return b;
}

static void die(const std::string &m)
{
    fprintf(stderr, "glioma_adaptive: %s\n", m.c_str());
    exit(2);
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

/* Each cell takes the dense voxel floor(x * n) at its vertex position, the
 * voxel lookup of the reference's _ic (Glioma_ReactionDiffusion.cpp:124-131). */
static void fill(GridT &grid)
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
                    const size_t g = (size_t)(int)floor(x[0] * g_n) +
                                     (size_t)g_n * ((int)floor(x[1] * g_n) + (size_t)g_n * (int)floor(x[2] * g_n));
                    block(ix, iy, iz).p_w = (Real)g_pw[g];
                    block(ix, iy, iz).p_g = (Real)g_pg[g];
                    block(ix, iy, iz).phi = (Real)g_phi[g];
                    block(ix, iy, iz).dphidt = 0;
                }
    }
}

/* FNV-1a over the sorted (level, ix, iy, iz) list of the leaves (the block
 * order of getBlocksInfo follows heap addresses, so lists are compared as
 * sorted sets). */
static unsigned long long leaves_hash(GridT &grid, int &nblocks)
{
    std::vector<BlockInfo> vInfo = grid.getBlocksInfo();
    std::vector<std::vector<int> > keys(vInfo.size(), std::vector<int>(4));
    for (size_t i = 0; i < vInfo.size(); i++) {
        keys[i][0] = vInfo[i].level;
        for (int d = 0; d < 3; d++) keys[i][1 + d] = vInfo[i].index[d];
    }
    std::sort(keys.begin(), keys.end());
    unsigned long long h = 1469598103934665603ull;
    for (size_t i = 0; i < keys.size(); i++)
        for (int q = 0; q < 4; q++)
            for (int b = 0; b < 4; b++) {
                h ^= ((unsigned)keys[i][q] >> (8 * b)) & 0xffu;
                h *= 1099511628211ull;
            }
    nblocks = (int)keys.size();
    return h;
}

static void write_finest(GridT &grid, int maxLevel, const char *path)
{
    const int n = g_n;
    std::vector<double> out((size_t)n * n * n, 0.0);
    std::vector<signed char> lev((size_t)n * n * n, -1);
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
                            for (int dx = 0; dx < r; dx++) {
                                const size_t q = (size_t)(x0 + dx) + (size_t)n * ((y0 + dy) + (size_t)n * (z0 + dz));
                                out[q] = v;
                                lev[q] = (signed char)info.level;
                            }
                }
    }
    FILE *f = fopen(path, "wb");
    if (!f) die("cannot write output");
    fwrite(&n, sizeof(int), 1, f);
    fwrite(&out[0], 8, out.size(), f);
    fclose(f);
    const std::string lp = std::string(path) + ".levels";
    f = fopen(lp.c_str(), "wb");
    if (!f) die("cannot write the level map");
    fwrite(&lev[0], 1, lev.size(), f);
    fclose(f);
}

int main(int argc, char **argv)
{
    if (argc != 8 && argc != 10)
        die("usage: glioma_adaptive <in.bin> <maxlevel> <refine_tol> <compress_tol> <nsteps> <every> <out.bin> "
            "[<Dw cm^2/day> <rho /day>]");
    read_dense(argv[1]);
    const int maxLevel = atoi(argv[2]);
    const double rtol = atof(argv[3]), ctol = atof(argv[4]);
    const int nsteps = atoi(argv[5]), every = atoi(argv[6]);
    if (g_n != 8 << maxLevel) die("the dense input must have 8 * 2^maxlevel cells per direction");
    if (every < 0 || nsteps < 0) die("bad arguments");
    const double Dw_day = argc == 10 ? atof(argv[8]) : 0.2, rho_day = argc == 10 ? atof(argv[9]) : 0.05;
    if (!(Dw_day > 0) || !(rho_day >= 0)) die("bad coefficients");

    try {
        Refiner_SpaceExtension refiner(1, maxLevel);
        Compressor compressor(1);
        GridT grid(4, 4, 4, maxStencil);
        grid.setRefiner(&refiner);
        grid.setCompressor(&compressor);
        fill(grid);
        BlockFWT<W, B, RD_Projector_Wavelets> blockfwt;
        Science::AutomaticRefinement<0, 0>(grid, blockfwt, rtol, maxLevel, -1, NULL, fill);
        Science::AutomaticCompression<0, 0>(grid, blockfwt, ctol, -1, NULL);

        const Real L = (Real)25.6;
        const Real Dw = (Real)((Real)Dw_day / (L * L));
        const Real Dg = (Real)(0.1 * Dw);
        const Real rho = (Real)rho_day;
        const Real h = (Real)(1. / (8 << maxLevel));
        const Real dt = (Real)(0.99 * h * h / (2. * 3 * (Dw >= Dg ? Dw : Dg)));

        std::vector<int> nblocks;
        std::vector<unsigned long long> hashes;
        int nb0 = 0;
        hashes.push_back(leaves_hash(grid, nb0));
        nblocks.push_back(nb0);

        /* room for every leaf of the finest level plus the children of a
         * split that coexist with their parents */
        const int capacity = (1 << (3 * maxLevel)) + (1 << (3 * maxLevel)) / 2;
        gbfk_mrag::ResidentGrid<GridT> rg(capacity);
        grid.setBlockSplitter(new gbfk_mrag::DeviceSplitter<W, BlockCollection<B>, GridT>(&rg));
        grid.setBlockCollapser(new gbfk_mrag::DeviceCollapser<W, BlockCollection<B>, GridT>(&rg));
        const double tu = gbfk_mrag::wall_seconds();
        rg.upload_all(grid);
        const double t_first_upload = gbfk_mrag::wall_seconds() - tu;

        double t_step = 0, t_adapt = 0;
        long long cell_updates = 0;
        int changes = 0;
        for (int done = 0; done < nsteps;) {
            const int k = every > 0 ? std::min(every, nsteps - done) : nsteps - done;
            const std::vector<BlockInfo> vInfo = rg.sync(grid);
            const double t0 = gbfk_mrag::wall_seconds();
            gbfk_mrag::ok(rg.ctx, gbfk_rd_step(rg.ctx, Dw, Dg, rho, dt, k, 1), "gbfk_rd_step");
            t_step += gbfk_mrag::wall_seconds() - t0;
            cell_updates += (long long)k * (long long)vInfo.size() * 512;
            done += k;
            if (every == 0) break;  // the set-up's grid for the whole run
            const double ta = gbfk_mrag::wall_seconds();
            rg.adaptation++;
            gbfk_mrag::AutomaticRefinement(grid, rg, rtol, maxLevel, 1);
            gbfk_mrag::AutomaticCompression(grid, rg, ctol, -1);
            t_adapt += gbfk_mrag::wall_seconds() - ta;
            int nb = 0;
            hashes.push_back(leaves_hash(grid, nb));
            if (hashes.back() != hashes[hashes.size() - 2]) changes++;
            nblocks.push_back(nb);
        }
        rg.download_phi(grid);
        write_finest(grid, maxLevel, argv[7]);

        const gbfk_mrag::ResidentStats &st = rg.stats;
        printf("{\"mode\": \"gpu\", \"real_bytes\": %d, \"maxlevel\": %d, \"steps\": %d, \"every\": %d, \"dt\": %.17g, "
               "\"step_seconds\": %.6f, \"adapt_seconds\": %.6f, \"first_upload_seconds\": %.6f, "
               "\"topology_changes\": %d, \"uploads\": %d, \"upload_seconds\": %.6f, \"detail_sweeps\": %d, "
               "\"details_seconds\": %.6f, \"plan_seconds\": %.6f, \"splits\": %d, \"split_seconds\": %.6f, "
               "\"collapses\": %d, \"collapse_seconds\": %.6f, \"cell_updates\": %lld, "
               "\"min_margin_refine\": %s, \"min_margin_compress\": %s, \"near_decisions\": %d, \"near\": [",
               (int)sizeof(Real), maxLevel, nsteps, every, (double)dt, t_step, t_adapt, t_first_upload, changes,
               st.uploads, st.t_upload, st.detail_sweeps, st.t_details, st.t_plan, st.splits, st.t_split,
               st.collapses, st.t_collapse, cell_updates, json_number(rg.min_margin_refine).c_str(),
               json_number(rg.min_margin_compress).c_str(),
               (int)rg.near.size());
        for (size_t i = 0; i < rg.near.size() && i < 200; i++) {
            const gbfk_mrag::NearDecision &d = rg.near[i];
            printf("%s[%d, %d, %d, %d, %d, %.17g, %.17g]", i ? ", " : "", d.adaptation, d.level, d.index[0],
                   d.index[1], d.index[2], d.detail, d.tol);
        }
        printf("], \"blocks\": [");
        for (size_t i = 0; i < nblocks.size(); i++) printf("%s%d", i ? ", " : "", nblocks[i]);
        printf("], \"hashes\": [");
        for (size_t i = 0; i < hashes.size(); i++) printf("%s\"%016llx\"", i ? ", " : "", hashes[i]);
        printf("]}\n");
    } catch (const gbfk_mrag::Error &e) {
        die(e.what());
    }
    return 0;
}
