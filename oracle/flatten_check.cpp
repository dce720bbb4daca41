/*
 * Host-side check of the adapter include/gbfk_mrag.hpp on the reference's own
 * MRAG grid.  Test infrastructure: compiled with the reference's unmodified
 * sources (oracle/Makefile, target ref); needs no GPU and calls nothing of
 * libgbfk.
 *
 *   flatten_check <maxlevel> <refine_tol> <compress_tol> <threads>
 *
 * Builds a level-2 grid (4^3 blocks, periodic, stencil [-1,2)), refines it
 * with Science::AutomaticRefinement up to <maxlevel> on analytic fields (a
 * Gaussian tumour, smooth tissue fractions, resampled after every
 * refinement) and compresses it once, then checks
 *  - gbfk_mrag::flatten_into with GBFK_HOST_THREADS = 1 and = <threads>
 *    against a plain serial restatement of the layout: blocks in vInfo
 *    order; per block its ghost rows in BlockLab::load order (icode 0..26
 *    without the block itself, 13, MRAG/MRAGcore/MRAGBlockLab.h:256-279);
 *    per entry the source leaf's slot * 512 + cell and the three weights;
 *  - flatten_into into a Topology that held larger, stale lists;
 *  - the shape gbfk_set_topology accepts: 488 rows per block, row_ptr
 *    non-decreasing from 0, every source in a leaf;
 *  - gather_anatomy against gather_into of each field, and scatter_from of
 *    the gathered phi leaving every Cell unchanged.
 * Prints one JSON line: leaves, entries, ok, the first failed check, and the
 * best of 5 timings (ms) of the serial restatement and of flatten_into at 1
 * and <threads> threads.
 */
#include <sys/time.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <string>
#include <vector>

#include "Glioma_Types.h"
#include "gbfk_mrag.hpp"

static int maxStencil[2][3] = {{-1, -1, -1}, {+2, +2, +2}};

static double now()
{
    timeval tv;
    gettimeofday(&tv, NULL);
    return tv.tv_sec + 1e-6 * tv.tv_usec;
}

static void fill(Grid<W, B> &grid)
{
    std::vector<BlockInfo> vInfo = grid.getBlocksInfo();
    const double pi = 3.14159265358979323846;
    for (size_t i = 0; i < vInfo.size(); i++) {
        const BlockInfo &info = vInfo[i];
        B &block = grid.getBlockCollection()[info.blockID];
        for (int iz = 0; iz < B::sizeZ; iz++)
            for (int iy = 0; iy < B::sizeY; iy++)
                for (int ix = 0; ix < B::sizeX; ix++) {
                    double x[3];
                    info.pos(x, ix, iy, iz);
                    const double r2 = (x[0] - 0.45) * (x[0] - 0.45) + (x[1] - 0.5) * (x[1] - 0.5) +
                                      (x[2] - 0.55) * (x[2] - 0.55);
                    const double pw = 0.5 + 0.4 * sin(2 * pi * x[0]) * cos(2 * pi * x[1]);
                    block(ix, iy, iz).p_w = (Real)pw;
                    block(ix, iy, iz).p_g = (Real)(0.9 - pw);
                    block(ix, iy, iz).phi = (Real)exp(-r2 / (2 * 0.04 * 0.04));
                    block(ix, iy, iz).dphidt = 0;
                }
    }
}

struct Flat {
    std::vector<int64_t> row_ptr, src;
    std::vector<double> w0, w1, w2;
};

/* The layout, written out one entry at a time. */
static Flat serial_flatten(const std::vector<BlockInfo> &vInfo, BoundaryInfo &bi)
{
    Flat f;
    std::map<int, int> slot;
    for (size_t i = 0; i < vInfo.size(); i++) slot[vInfo[i].blockID] = (int)i;
    f.row_ptr.push_back(0);
    for (size_t i = 0; i < vInfo.size(); i++) {
        BoundaryInfoBlock &bb = *bi.boundaryInfoOfBlock[vInfo[i].blockID];
        bb.lock();
        for (int icode = 0; icode < 27; icode++) {
            if (icode == 13) continue;
            for (unsigned g = 0; g < bb.boundary[icode].nGhosts; g++) {
                const std::vector<IndexWP> &row = bb.getGhosts()[bb.boundary[icode].start + g];
                for (size_t k = 0; k < row.size(); k++) {
                    const PointIndex &p = bb.getIndexPool()[row[k].point_index];
                    f.src.push_back((int64_t)slot[p.blockID] * 512 + p.index);
                    f.w0.push_back(bb.weightsPool[row[k].weights_index[0]]);
                    f.w1.push_back(bb.weightsPool[row[k].weights_index[1]]);
                    f.w2.push_back(bb.weightsPool[row[k].weights_index[2]]);
                }
                f.row_ptr.push_back((int64_t)f.src.size());
            }
        }
        bb.release();
    }
    return f;
}

static std::string failed;

static void expect(bool ok, const char *what)
{
    if (!ok && failed.empty()) failed = what;
}

static bool same(const Flat &f, const gbfk_mrag::Topology &t, const std::vector<BlockInfo> &vInfo)
{
    if (t.blocks.size() != vInfo.size()) return false;
    for (size_t i = 0; i < vInfo.size(); i++) {
        const gbfk_blockinfo &b = t.blocks[i];
        if (b.slot != (int)i || b.level != vInfo[i].level || b.h != (double)vInfo[i].h[0]) return false;
        for (int d = 0; d < 3; d++)
            if (b.index[d] != vInfo[i].index[d]) return false;
        if (t.slot_of[vInfo[i].blockID] != (int)i) return false;
    }
    return f.row_ptr == t.row_ptr && f.src == t.src && f.w0 == t.w0 && f.w1 == t.w1 && f.w2 == t.w2;
}

int main(int argc, char **argv)
{
    if (argc != 5) {
        fprintf(stderr, "usage: flatten_check <maxlevel> <refine_tol> <compress_tol> <threads>\n");
        return 2;
    }
    const int maxLevel = atoi(argv[1]);
    const double rtol = atof(argv[2]), ctol = atof(argv[3]);
    const std::string threads = argv[4];

    Refiner_SpaceExtension refiner(1, maxLevel);
    Compressor compressor(1);
    Grid<W, B> grid(4, 4, 4, maxStencil);
    grid.setRefiner(&refiner);
    grid.setCompressor(&compressor);
    fill(grid);
    BlockFWT<W, B, RD_Projector_Wavelets> blockfwt;
    Science::AutomaticRefinement<0, 0>(grid, blockfwt, rtol, maxLevel, -1, NULL, fill);
    Science::AutomaticCompression<0, 0>(grid, blockfwt, ctol, -1, NULL);
    std::vector<BlockInfo> vInfo = grid.getBlocksInfo();
    BoundaryInfo &bi = grid.getBoundaryInfo();
    const size_t nb = vInfo.size();

    double t_serial = 1e30, t_one = 1e30, t_many = 1e30;
    Flat ref;
    for (int r = 0; r < 5; r++) {
        const double t0 = now();
        ref = serial_flatten(vInfo, bi);
        t_serial = std::min(t_serial, now() - t0);
    }

    gbfk_mrag::Topology t;
    /* stale, larger lists first: flatten_into must overwrite or drop them */
    t.blocks.resize(2 * nb + 3);
    t.slot_of.assign(5, 7);
    t.row_ptr.assign(2 * ref.row_ptr.size() + 5, -3);
    t.src.assign(2 * ref.src.size() + 5, -5);
    t.w0.assign(t.src.size(), -1.0);
    t.w1.assign(t.src.size(), -1.0);
    t.w2.assign(t.src.size(), -1.0);
    setenv("GBFK_HOST_THREADS", "1", 1);
    for (int r = 0; r < 5; r++) {
        const double t0 = now();
        gbfk_mrag::flatten_into(t, vInfo, bi);
        t_one = std::min(t_one, now() - t0);
        expect(same(ref, t, vInfo), "flatten_into, 1 thread");
    }
    setenv("GBFK_HOST_THREADS", threads.c_str(), 1);
    for (int r = 0; r < 5; r++) {
        const double t0 = now();
        gbfk_mrag::flatten_into(t, vInfo, bi);
        t_many = std::min(t_many, now() - t0);
        expect(same(ref, t, vInfo), "flatten_into, many threads");
    }
    expect(same(ref, gbfk_mrag::flatten(vInfo, bi), vInfo), "flatten");

    expect(t.row_ptr.size() == nb * GBFK_LAB_GHOSTS + 1, "488 rows per block");
    expect(!t.row_ptr.empty() && t.row_ptr[0] == 0, "row_ptr starts at 0");
    for (size_t r = 0; r + 1 < t.row_ptr.size(); r++) expect(t.row_ptr[r] <= t.row_ptr[r + 1], "row_ptr monotone");
    for (size_t k = 0; k < t.src.size(); k++)
        expect(t.src[k] >= 0 && t.src[k] < (int64_t)nb * GBFK_BLOCK_CELLS, "sources in leaves");

    typedef B::ElementType Cell;
    std::vector<Real> pw, pg, phi, pw1, pg1, phi1, phi2;
    gbfk_mrag::gather_anatomy(pw, pg, phi, grid.getBlockCollection(), vInfo);
    gbfk_mrag::gather_into(pw1, grid.getBlockCollection(), vInfo, gbfk_mrag::get_pw<Cell>());
    gbfk_mrag::gather_into(pg1, grid.getBlockCollection(), vInfo, gbfk_mrag::get_pg<Cell>());
    gbfk_mrag::gather_into(phi1, grid.getBlockCollection(), vInfo, gbfk_mrag::get_phi<Cell>());
    expect(pw == pw1 && pg == pg1 && phi == phi1, "gather_anatomy = gather_into");
    bool ordered = phi.size() == nb * GBFK_BLOCK_CELLS;
    for (size_t i = 0; i < nb && ordered; i++) {
        B &block = grid.getBlockCollection()[vInfo[i].blockID];
        for (int c = 0; c < GBFK_BLOCK_CELLS; c++)
            if (phi[i * GBFK_BLOCK_CELLS + c] != block(c % 8, (c / 8) % 8, c / 64).phi) ordered = false;
    }
    expect(ordered, "gathered cells slot-major, x fastest");
    for (size_t k = 0; k < phi.size(); k++) phi1[k] = (Real)(k % 977);
    gbfk_mrag::scatter_from(phi1, grid.getBlockCollection(), vInfo, gbfk_mrag::set_phi<Cell>());
    gbfk_mrag::gather_into(phi2, grid.getBlockCollection(), vInfo, gbfk_mrag::get_phi<Cell>());
    expect(phi2 == phi1, "scatter_from then gather_into");
    gbfk_mrag::scatter_from(phi, grid.getBlockCollection(), vInfo, gbfk_mrag::set_phi<Cell>());

    printf("{\"leaves\": %d, \"entries\": %lld, \"threads\": %s, \"ok\": %s, \"failed\": \"%s\", "
           "\"serial_ms\": %.3f, \"flatten_1_ms\": %.3f, \"flatten_n_ms\": %.3f}\n",
           (int)nb, (long long)ref.src.size(), threads.c_str(), failed.empty() ? "true" : "false", failed.c_str(),
           t_serial * 1e3, t_one * 1e3, t_many * 1e3);
    return failed.empty() ? 0 : 1;
}
