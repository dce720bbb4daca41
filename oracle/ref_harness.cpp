/*
 * Oracle harness around the reference's own Fisher-Kolmogorov operators.
 *
 * Test infrastructure only: this file is compiled together with the
 * reference's unmodified MRAG/Glioma sources (see oracle/Makefile) into
 * oracle/_ref/ref_harness_{f64,f32}.  It drives the reference code exactly as
 * Glioma_ReactionDiffusion::_reactionDiffusionStep does
 * (Glioma/Glioma_ReactionDiffusion.cpp:176-187): one
 * BlockProcessing::pipeline_process with ReactionDiffusionOperator<3>
 * followed by BlockProcessing::process with UpdateTumor<3>, on an MRAG Grid
 * whose fields were written cell by cell from a dense input.  It bypasses
 * run()'s forced refine/compress (Glioma_ReactionDiffusion.cpp:312-313) so
 * that a uniform grid stays uniform.
 *
 * Modes
 *   uniform <in> <out> <Dw> <Dg> <rho> <dt> <nsteps>
 *       in : int32 n, then p_w[n^3], p_g[n^3], phi[n^3] as float64, x fastest
 *       out: phi[n^3] as float64 after nsteps steps
 *   rhs <in> <out> <Dw> <Dg> <rho>
 *       out: dphidt[n^3] as float64 of one ReactionDiffusionOperator sweep
 *   time <in> <Dw> <Dg> <rho> <dt> <nsteps> [nwarmup]
 *       runs nwarmup untimed steps, then times nsteps steps of the stepping
 *       loop only and prints one JSON line
 *   adapt ...  (see adapt_main below)
 * Dw and Dg are the already rescaled coefficients (Dw/L^2 and 0.1*Dw/L^2 in
 * Glioma_ReactionDiffusion.cpp:302-303).
 */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <vector>
#include <map>
#include <set>
#include <string>
#include <algorithm>
#include <iostream>
#include <fstream>
#include <sys/time.h>

#include "Glioma_Types.h"

static int maxStencil[2][3] = {
    {-1, -1, -1},
    {+2, +2, +2}
};

static double wall_seconds()
{
    struct timeval tv;
    gettimeofday(&tv, NULL);
    return tv.tv_sec + 1e-6 * tv.tv_usec;
}

struct Dense {
    int n;
    std::vector<double> pw, pg, phi;
};

static void die(const char *msg)
{
    fprintf(stderr, "ref_harness: %s\n", msg);
    exit(2);
}

static Dense read_dense(const char *path)
{
    Dense d;
    FILE *f = fopen(path, "rb");
    if (!f) die("cannot open input");
    int n = 0;
    if (fread(&n, sizeof(int), 1, f) != 1 || n <= 0 || n % _BLOCKSIZE_) die("bad header");
    d.n = n;
    const size_t N = (size_t)n * n * n;
    d.pw.resize(N); d.pg.resize(N); d.phi.resize(N);
    if (fread(&d.pw[0], sizeof(double), N, f) != N) die("short p_w");
    if (fread(&d.pg[0], sizeof(double), N, f) != N) die("short p_g");
    if (fread(&d.phi[0], sizeof(double), N, f) != N) die("short phi");
    fclose(f);
    return d;
}

static void write_doubles(const char *path, const std::vector<double> &v)
{
    FILE *f = fopen(path, "wb");
    if (!f) die("cannot open output");
    if (fwrite(&v[0], sizeof(double), v.size(), f) != v.size()) die("short write");
    fclose(f);
}

/* Copy the dense fields into the blocks of a uniform grid. */
static void fill_uniform(Grid<W, B> &grid, const Dense &d)
{
    const int n = d.n;
    std::vector<BlockInfo> vInfo = grid.getBlocksInfo();
    for (size_t i = 0; i < vInfo.size(); i++) {
        const BlockInfo &info = vInfo[i];
        B &block = grid.getBlockCollection()[info.blockID];
        for (int iz = 0; iz < B::sizeZ; iz++)
            for (int iy = 0; iy < B::sizeY; iy++)
                for (int ix = 0; ix < B::sizeX; ix++) {
                    const size_t gx = info.index[0] * B::sizeX + ix;
                    const size_t gy = info.index[1] * B::sizeY + iy;
                    const size_t gz = info.index[2] * B::sizeZ + iz;
                    const size_t g = gx + n * (gy + n * gz);
                    block(ix, iy, iz).p_w = (Real)d.pw[g];
                    block(ix, iy, iz).p_g = (Real)d.pg[g];
                    block(ix, iy, iz).phi = (Real)d.phi[g];
                    block(ix, iy, iz).dphidt = 0;
                }
    }
}

template <typename Getter>
static std::vector<double> gather_uniform(Grid<W, B> &grid, int n, Getter get)
{
    std::vector<double> out((size_t)n * n * n, 0.0);
    std::vector<BlockInfo> vInfo = grid.getBlocksInfo();
    for (size_t i = 0; i < vInfo.size(); i++) {
        const BlockInfo &info = vInfo[i];
        B &block = grid.getBlockCollection()[info.blockID];
        for (int iz = 0; iz < B::sizeZ; iz++)
            for (int iy = 0; iy < B::sizeY; iy++)
                for (int ix = 0; ix < B::sizeX; ix++) {
                    const size_t gx = info.index[0] * B::sizeX + ix;
                    const size_t gy = info.index[1] * B::sizeY + iy;
                    const size_t gz = info.index[2] * B::sizeZ + iz;
                    out[gx + n * (gy + n * gz)] = (double)get(block(ix, iy, iz));
                }
    }
    return out;
}

static double get_phi(const Cell &c) { return (double)c.phi; }
static double get_dphidt(const Cell &c) { return (double)c.dphidt; }

/* One step exactly as Glioma_ReactionDiffusion::_reactionDiffusionStep. */
static void rd_step(Grid<W, B> &grid, BlockProcessing &blockProcessing, BoundaryInfo *boundaryInfo,
                    int nParallelGranularity, Real Dw, Real Dg, Real rho, double dt)
{
    std::vector<BlockInfo> vInfo = grid.getBlocksInfo();
    const BlockCollection<B> &collecton = grid.getBlockCollection();
    ReactionDiffusionOperator<_DIM> rhs(Dw, Dg, rho);
    UpdateTumor<_DIM> updateTumor(dt);
    blockProcessing.pipeline_process(vInfo, collecton, *boundaryInfo, rhs);
    BlockProcessing::process(vInfo, collecton, updateTumor, nParallelGranularity);
}

static int uniform_main(int argc, char **argv, int mode)
{
    /* mode 0: uniform, 1: rhs, 2: time */
    const char *in = argv[2];
    int a = 3;
    const char *out = NULL;
    if (mode != 2) out = argv[a++];
    const Real Dw = (Real)atof(argv[a++]);
    const Real Dg = (Real)atof(argv[a++]);
    const Real rho = (Real)atof(argv[a++]);
    double dt = 0;
    int nsteps = 0, nwarmup = 0;
    if (mode != 1) {
        dt = atof(argv[a++]);
        nsteps = atoi(argv[a++]);
    }
    if (mode == 2 && a < argc) nwarmup = atoi(argv[a++]);

    Dense d = read_dense(in);
    const int bpd = d.n / B::sizeX;
    Grid<W, B> *grid = new Grid<W, B>(bpd, bpd, bpd, maxStencil);
    fill_uniform(*grid, d);
    BlockProcessing *blockProcessing = new BlockProcessing();
    BoundaryInfo *boundaryInfo = &grid->getBoundaryInfo();
    const int nParallelGranularity = (grid->getBlocksInfo().size() <= 8 ? 1 : 4);

    if (mode == 1) {
        std::vector<BlockInfo> vInfo = grid->getBlocksInfo();
        ReactionDiffusionOperator<_DIM> rhs(Dw, Dg, rho);
        blockProcessing->pipeline_process(vInfo, grid->getBlockCollection(), *boundaryInfo, rhs);
        write_doubles(out, gather_uniform(*grid, d.n, get_dphidt));
        return 0;
    }

    for (int s = 0; s < nwarmup; s++)
        rd_step(*grid, *blockProcessing, boundaryInfo, nParallelGranularity, Dw, Dg, rho, dt);
    const double t0 = wall_seconds();
    for (int s = 0; s < nsteps; s++)
        rd_step(*grid, *blockProcessing, boundaryInfo, nParallelGranularity, Dw, Dg, rho, dt);
    const double t1 = wall_seconds();

    if (mode == 0) {
        write_doubles(out, gather_uniform(*grid, d.n, get_phi));
    } else {
        const double cells = (double)d.n * d.n * d.n;
        printf("{\"cells\": %.0f, \"steps\": %d, \"seconds\": %.6f, \"threads\": %d, "
               "\"real_bytes\": %d, \"cell_updates_per_s\": %.6e}\n",
               cells, nsteps, t1 - t0, tbb::task_scheduler_init::default_num_threads(),
               (int)sizeof(Real), cells * nsteps / (t1 - t0));
    }
    return 0;
}

int main(int argc, char **argv)
{
    if (argc < 2) die("usage: ref_harness uniform|rhs|time ...");
    std::string mode = argv[1];
    if (mode == "uniform" && argc == 9) return uniform_main(argc, argv, 0);
    if (mode == "rhs" && argc == 7) return uniform_main(argc, argv, 1);
    if (mode == "time" && (argc == 8 || argc == 9)) return uniform_main(argc, argv, 2);
    die("bad arguments");
    return 2;
}
