/*
 * The reference's own wavelet details, block split and block collapse on an
 * adapted MRAG grid: the values the oracle's fwt_detail_pool, split_block
 * and collapse_blocks restate.  Test infrastructure: compiled with the
 * reference's unmodified sources (oracle/Makefile, target ref); no GPU.
 *
 *   topo_harness <base_bpd> <maxlevel> <refine_tol> <every> <out.bin>
 *
 * A grid of base_bpd^3 blocks (periodic, stencil [-1,2), as the RD operator
 * needs) is refined with Science::AutomaticRefinement up to maxlevel - 1 on
 * analytic fields (a Gaussian tumour, smooth tissue fractions and a ball of
 * CSF without tissue, each value rounded to a multiple of 2^-10 so that the
 * dump compresses; resampled after every refinement).  Then, on that grid:
 *  - rhs: one sweep of the reference's ReactionDiffusionOperator through
 *    BlockProcessing::pipeline_process (Glioma_ReactionDiffusion.cpp:176-183;
 *    Dw = 0.2 cm^2/day on L = 25.6 cm, Dg = Dw/10, rho = 0.05/day): dphidt of
 *    every leaf, with each leaf's h and the three coefficients in Real;
 *  - detail: BlockFWT::multichannel_fwt<0,0> (MRAG/MRAGcore/MRAGBlockFWT.h,
 *    the per-block detail AutomaticRefinement compares with its tolerance,
 *    MRAG/MRAGscience/MRAGScienceCore.h:68-79) of every leaf;
 *  - split: Grid::refine (MRAG/MRAGcore/MRAGrid.inl:248-280, the
 *    BlockSplitter on the pre-refinement ghosts) of every <every>-th leaf
 *    below maxlevel (the refiner may add neighbours); each refined parent's
 *    eight children, child c = cx + 2 (cy + 2 cz);
 *  - collapse: Grid::compress of all those children; each parent that came
 *    back, its cells.
 * The dump holds, for the grid before the split: the leaves (level, index)
 * in vInfo order, the ghost lists flattened by include/gbfk_mrag.hpp, p_w,
 * p_g, phi slot-major (512 per leaf, x fastest), rhs, h, the coefficients,
 * the details; then the split
 * parents' slots with their children's fields, and the collapsed parents
 * (their positions in the split list) with their fields.  Format: records of
 * int32 name length, name, int32 kind (0 int64, 1 float64), int64 count,
 * data.
 */
#include <sys/time.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <set>
#include <string>
#include <vector>

#include "Glioma_Types.h"
#include "gbfk_mrag.hpp"

static int maxStencil[2][3] = {{-1, -1, -1}, {+2, +2, +2}};

static double q10(double v) { return floor(v * 1024.0 + 0.5) / 1024.0; }

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
                    const double r2 = (x[0] - 0.42) * (x[0] - 0.42) + (x[1] - 0.55) * (x[1] - 0.55) +
                                      (x[2] - 0.5) * (x[2] - 0.5);
                    const double pw = 0.5 + 0.45 * sin(2 * pi * x[0]) * cos(2 * pi * x[2]);
                    const double c2 = (x[0] - 0.62) * (x[0] - 0.62) + (x[1] - 0.5) * (x[1] - 0.5) +
                                      (x[2] - 0.45) * (x[2] - 0.45);
                    const bool csf = c2 < 0.09 * 0.09; /* a ventricle: no tissue, no flux */
                    block(ix, iy, iz).p_w = csf ? (Real)0 : (Real)q10(pw);
                    block(ix, iy, iz).p_g = csf ? (Real)0 : (Real)q10(0.95 - pw);
                    block(ix, iy, iz).phi = (Real)q10(exp(-r2 / (2 * 0.07 * 0.07)));
                    block(ix, iy, iz).dphidt = 0;
                }
    }
}

static void put_i(FILE *f, const char *name, const std::vector<int64_t> &v)
{
    const int len = (int)strlen(name), kind = 0;
    const int64_t n = (int64_t)v.size();
    fwrite(&len, 4, 1, f);
    fwrite(name, 1, len, f);
    fwrite(&kind, 4, 1, f);
    fwrite(&n, 8, 1, f);
    if (n) fwrite(&v[0], 8, n, f);
}

static void put_d(FILE *f, const char *name, const std::vector<double> &v)
{
    const int len = (int)strlen(name), kind = 1;
    const int64_t n = (int64_t)v.size();
    fwrite(&len, 4, 1, f);
    fwrite(name, 1, len, f);
    fwrite(&kind, 4, 1, f);
    fwrite(&n, 8, 1, f);
    if (n) fwrite(&v[0], 8, n, f);
}

typedef B::ElementType Cell;

struct get_dphidt {
    Real operator()(const Cell &c) const { return c.dphidt; }
};

static void put_fields(FILE *f, const std::string &prefix, Grid<W, B> &grid, const std::vector<BlockInfo> &blocks)
{
    std::vector<Real> a;
    const char *names[3] = {"p_w", "p_g", "phi"};
    for (int k = 0; k < 3; k++) {
        if (k == 0) gbfk_mrag::gather_into(a, grid.getBlockCollection(), blocks, gbfk_mrag::get_pw<Cell>());
        if (k == 1) gbfk_mrag::gather_into(a, grid.getBlockCollection(), blocks, gbfk_mrag::get_pg<Cell>());
        if (k == 2) gbfk_mrag::gather_into(a, grid.getBlockCollection(), blocks, gbfk_mrag::get_phi<Cell>());
        put_d(f, (prefix + names[k]).c_str(), std::vector<double>(a.begin(), a.end()));
    }
}

static long long key(int level, int x, int y, int z)
{
    return (((long long)level * 4096 + z) * 4096 + y) * 4096 + x;
}

static long long key(const BlockInfo &b) { return key(b.level, b.index[0], b.index[1], b.index[2]); }

int main(int argc, char **argv)
{
    if (argc != 6) {
        fprintf(stderr, "usage: topo_harness <base_bpd> <maxlevel> <refine_tol> <every> <out.bin>\n");
        return 2;
    }
    const int bpd = atoi(argv[1]), maxLevel = atoi(argv[2]), every = atoi(argv[4]);
    const double rtol = atof(argv[3]);
    if (bpd < 1 || maxLevel < 1 || every < 1) return 2;

    Refiner_SpaceExtension refiner(1, maxLevel);
    Compressor compressor(1);
    Grid<W, B> grid(bpd, bpd, bpd, maxStencil);
    grid.setRefiner(&refiner);
    grid.setCompressor(&compressor);
    fill(grid);
    BlockFWT<W, B, RD_Projector_Wavelets> blockfwt;
    Science::AutomaticRefinement<0, 0>(grid, blockfwt, rtol, maxLevel - 1, -1, NULL, fill);

    std::vector<BlockInfo> vInfo = grid.getBlocksInfo();
    const size_t nb = vInfo.size();
    FILE *f = fopen(argv[5], "wb");
    if (!f) return 2;

    std::vector<int64_t> lv, ix;
    for (size_t i = 0; i < nb; i++) {
        lv.push_back(vInfo[i].level);
        for (int d = 0; d < 3; d++) ix.push_back(vInfo[i].index[d]);
    }
    put_i(f, "level", lv);
    put_i(f, "index", ix);
    gbfk_mrag::Topology t = gbfk_mrag::flatten(vInfo, grid.getBoundaryInfo());
    put_i(f, "row_ptr", t.row_ptr);
    put_i(f, "src", t.src);
    put_d(f, "w0", t.w0);
    put_d(f, "w1", t.w1);
    put_d(f, "w2", t.w2);
    put_fields(f, "", grid, vInfo);

    /* one ReactionDiffusionOperator sweep (Glioma_ReactionDiffusion.cpp:176-183):
     * dphidt of every leaf, with its spacing and the coefficients */
    {
        const Real L = (Real)25.6;
        const Real Dw = (Real)((Real)0.2 / (L * L)), Dg = (Real)(0.1 * Dw), rho = (Real)0.05;
        ReactionDiffusionOperator<_DIM> rhs(Dw, Dg, rho);
        BlockProcessing bp;
        bp.pipeline_process(vInfo, grid.getBlockCollection(), grid.getBoundaryInfo(), rhs);
        std::vector<Real> a;
        gbfk_mrag::gather_into(a, grid.getBlockCollection(), vInfo, get_dphidt());
        put_d(f, "rhs", std::vector<double>(a.begin(), a.end()));
        std::vector<double> h(nb), coeffs(3);
        for (size_t i = 0; i < nb; i++) h[i] = (double)vInfo[i].h[0];
        coeffs[0] = (double)Dw;
        coeffs[1] = (double)Dg;
        coeffs[2] = (double)rho;
        put_d(f, "h", h);
        put_d(f, "coeffs", coeffs);
    }

    std::vector<FWTReport<1> > rep =
        BlockFWT<W, B, RD_Projector_Wavelets>::multichannel_fwt<0, 0>(vInfo, grid.getBlockCollection(),
                                                                       grid.getBoundaryInfo());
    std::vector<double> det(nb);
    for (size_t i = 0; i < nb; i++) det[i] = rep[i].getOverAll_DetailMaxMag();
    put_d(f, "detail", det);

    std::set<int> to_refine;
    for (size_t i = 0; i < nb; i += every)
        if (vInfo[i].level < maxLevel) to_refine.insert(vInfo[i].blockID);
    grid.refine(to_refine);
    grid.getBoundaryInfo();

    std::vector<BlockInfo> after = grid.getBlocksInfo();
    std::set<int> alive;
    for (size_t i = 0; i < after.size(); i++) alive.insert(after[i].blockID);
    std::map<long long, BlockInfo> leaf_at;
    for (size_t i = 0; i < after.size(); i++) leaf_at[key(after[i])] = after[i];

    std::vector<int64_t> parents;
    std::vector<BlockInfo> children;
    std::set<int> child_ids;
    for (size_t i = 0; i < nb; i++) {
        if (alive.count(vInfo[i].blockID)) continue;
        std::vector<BlockInfo> kids;
        for (int c = 0; c < 8; c++) {
            int ci[3];
            for (int d = 0; d < 3; d++) ci[d] = 2 * vInfo[i].index[d] + ((c >> d) & 1);
            std::map<long long, BlockInfo>::const_iterator it = leaf_at.find(key(vInfo[i].level + 1, ci[0], ci[1], ci[2]));
            if (it == leaf_at.end()) break;
            kids.push_back(it->second);
        }
        if (kids.size() != 8) {
            fprintf(stderr, "topo_harness: block %d vanished without eight leaf children\n", vInfo[i].blockID);
            return 1;
        }
        parents.push_back((int64_t)i);
        for (int c = 0; c < 8; c++) {
            children.push_back(kids[c]);
            child_ids.insert(kids[c].blockID);
        }
    }
    put_i(f, "split_parent", parents);
    put_fields(f, "split_", grid, children);

    int ncollapsed = 0;
    grid.compress(child_ids, ncollapsed);
    grid.getBoundaryInfo();
    std::vector<BlockInfo> back = grid.getBlocksInfo();
    std::map<long long, BlockInfo> back_at;
    for (size_t i = 0; i < back.size(); i++) back_at[key(back[i])] = back[i];
    std::vector<int64_t> collapsed;
    std::vector<BlockInfo> restored;
    for (size_t p = 0; p < parents.size(); p++) {
        const BlockInfo &old = vInfo[parents[p]];
        std::map<long long, BlockInfo>::const_iterator it = back_at.find(key(old));
        if (it == back_at.end()) continue;
        collapsed.push_back((int64_t)p);
        restored.push_back(it->second);
    }
    put_i(f, "collapse_parent", collapsed);
    put_fields(f, "collapse_", grid, restored);
    fclose(f);
    printf("{\"leaves\": %d, \"split\": %d, \"collapsed\": %d, \"entries\": %lld, \"real_bytes\": %d}\n", (int)nb,
           (int)parents.size(), (int)collapsed.size(), (long long)t.src.size(), (int)sizeof(Real));
    return 0;
}
