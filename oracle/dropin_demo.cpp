/*
 * Drop-in check on adaptive grids built by the reference's own MRAG code.
 *
 * Test infrastructure: compiled with the reference's unmodified sources and
 * the adapter include/gbfk_mrag.hpp, linked against libgbfk.so (see
 * oracle/Makefile, target dropin).  It needs a GPU at run time.
 *
 *   dropin_demo <in.bin> <maxlevel> <refine_tol> <steps>
 *
 * 1. Builds a level-2 grid (4^3 blocks, periodic, stencil [-1,2)) and refines
 *    it with the reference's Science::AutomaticRefinement (MRAGScienceCore.h:
 *    42-108) up to <maxlevel>, resampling p_w, p_g, phi from the dense input
 *    after every refinement (the fillGrid hook), so the leaves span several
 *    levels with the reference's own coarse-fine ghost lists.
 * 2. Wavelet details: BlockFWT::multichannel_fwt<0,0> (MRAGBlockFWT.h:447-478)
 *    vs gbfk_fwt_details, per block.
 * 3. RD steps: <steps> steps of the reference's pipeline_process/process
 *    (Glioma_ReactionDiffusion.cpp:176-187, threaded TBB stand-in) vs the same
 *    two calls on gbfk_mrag::BlockProcessing_CUDA (the drop-in policy) and vs
 *    one gbfk_rd_step(steps) call with the data resident on the GPU.
 * 4. Split: the reference's Grid::refine on the blocks with the largest
 *    details vs gbfk_split on the pre-refinement topology, per child.
 * 5. Collapse: the reference's Grid::compress on one family of siblings vs
 *    gbfk_collapse.
 * Prints one JSON line with the mismatch counts (all must be 0).
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

static int g_n = 0;
static std::vector<double> g_pw, g_pg, g_phi;

static void die(const char *m)
{
    fprintf(stderr, "dropin_demo: %s\n", m);
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

/* p_w, p_g, phi of every cell sampled from the dense volume at the cell's
 * vertex position, as the reference's _ic maps anatomy voxels
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

typedef std::map<int, std::vector<Real> > FieldMap; /* blockID -> 512 values */

static FieldMap snapshot(Grid<W, B> &grid, int which)
{
    FieldMap m;
    std::vector<BlockInfo> vInfo = grid.getBlocksInfo();
    for (size_t i = 0; i < vInfo.size(); i++) {
        B &block = grid.getBlockCollection()[vInfo[i].blockID];
        std::vector<Real> v;
        for (int iz = 0; iz < 8; iz++)
            for (int iy = 0; iy < 8; iy++)
                for (int ix = 0; ix < 8; ix++)
                    v.push_back(which == 0 ? block(ix, iy, iz).phi : which == 1 ? block(ix, iy, iz).p_w
                                                                                : block(ix, iy, iz).p_g);
        m[vInfo[i].blockID] = v;
    }
    return m;
}

static void restore_phi(Grid<W, B> &grid, const FieldMap &m)
{
    std::vector<BlockInfo> vInfo = grid.getBlocksInfo();
    for (size_t i = 0; i < vInfo.size(); i++) {
        B &block = grid.getBlockCollection()[vInfo[i].blockID];
        const std::vector<Real> &v = m.find(vInfo[i].blockID)->second;
        int k = 0;
        for (int iz = 0; iz < 8; iz++)
            for (int iy = 0; iy < 8; iy++)
                for (int ix = 0; ix < 8; ix++) block(ix, iy, iz).phi = v[k++];
    }
}

static double now()
{
    timeval tv;
    gettimeofday(&tv, NULL);
    return tv.tv_sec + 1e-6 * tv.tv_usec;
}

static long count_diff(const std::vector<Real> &a, const Real *b, int n)
{
    long d = 0;
    for (int i = 0; i < n; i++)
        if (memcmp(&a[i], &b[i], sizeof(Real)) != 0) d++;
    return d;
}

template <typename BP>
static void rd_step(Grid<W, B> &grid, BP &bp, Real Dw, Real Dg, Real rho, double dt)
{
    /* the two calls of Glioma_ReactionDiffusion::_reactionDiffusionStep */
    std::vector<BlockInfo> vInfo = grid.getBlocksInfo();
    const BlockCollection<B> &collecton = grid.getBlockCollection();
    ReactionDiffusionOperator<_DIM> rhs(Dw, Dg, rho);
    UpdateTumor<_DIM> updateTumor(dt);
    bp.pipeline_process(vInfo, collecton, grid.getBoundaryInfo(), rhs);
    BP::process(vInfo, collecton, updateTumor, 4);
}

int main(int argc, char **argv)
{
    if (argc != 5) die("usage: dropin_demo <in.bin> <maxlevel> <refine_tol> <steps>");
    read_dense(argv[1]);
    const int maxLevel = atoi(argv[2]);
    const double tol = atof(argv[3]);
    const int steps = atoi(argv[4]);
    if (g_n != 8 << maxLevel) die("the dense input must have 8 * 2^maxlevel cells per direction");

    Refiner_SpaceExtension refiner(1, maxLevel);
    Compressor compressor(1);
    Grid<W, B> grid(4, 4, 4, maxStencil);
    grid.setRefiner(&refiner);
    grid.setCompressor(&compressor);
    fill(grid);
    BlockFWT<W, B, RD_Projector_Wavelets> blockfwt;
    Science::AutomaticRefinement<0, 0>(grid, blockfwt, tol, maxLevel, -1, NULL, fill);

    std::vector<BlockInfo> vInfo = grid.getBlocksInfo();
    const int nb = (int)vInfo.size();
    std::map<int, int> levels;
    for (int i = 0; i < nb; i++) levels[vInfo[i].level]++;

    /* Dw = 0.2 cm^2/day on L = 25.6 cm, rho = 0.05/day, the CFL dt of the
     * finest level (Glioma_ReactionDiffusion.cpp:302-307 with h of maxlevel) */
    const Real L = (Real)25.6;
    const Real Dw = (Real)((Real)0.2 / (L * L));
    const Real Dg = (Real)(0.1 * Dw);
    const Real rho = (Real)0.05;
    const Real h = (Real)(1. / (8 << maxLevel));
    const Real dt = (Real)(0.99 * h * h / (2. * 3 * (Dw >= Dg ? Dw : Dg)));

    gbfk_mrag::Device dev(4 * nb + 64);

    /* 2. wavelet details */
    long fwt_mismatch = 0;
    double fwt_max = 0;
    {
        std::vector<FWTReport<1> > rep = BlockFWT<W, B, RD_Projector_Wavelets>::multichannel_fwt<0, 0>(
            vInfo, grid.getBlockCollection(), grid.getBoundaryInfo());
        dev.upload(vInfo, grid.getBlockCollection(), grid.getBoundaryInfo());
        std::vector<double> d(nb);
        gbfk_mrag::check(dev.ctx, gbfk_fwt_details(dev.ctx, &d[0]), "gbfk_fwt_details");
        for (int i = 0; i < nb; i++) {
            const double r = rep[i].getOverAll_DetailMaxMag();
            if (memcmp(&r, &d[i], sizeof(double)) != 0) fwt_mismatch++;
            fwt_max = std::max(fwt_max, r);
        }
    }

    /* 3. RD steps: the reference's step loop, the same loop through the drop-in
     * policy (write-back after every step, then deferred to sync_host), and one
     * resident gbfk_rd_step call */
    long step_mismatch_dropin = 0, step_mismatch_deferred = 0, step_mismatch_resident = 0;
    int n_ghost_faces = 0;
    double t_ref = 0, t_dropin = 0, t_deferred = 0;
    long dropin_uploads = 0;
    {
        typedef gbfk_mrag::BlockProcessing_CUDA<B> Policy;
        FieldMap phi0 = snapshot(grid, 0);
        BlockProcessing ref;
        double t0 = now();
        for (int s = 0; s < steps; s++) rd_step(grid, ref, Dw, Dg, rho, dt);
        t_ref = now() - t0;
        FieldMap phi_ref = snapshot(grid, 0);

        restore_phi(grid, phi0);
        Policy gpu;
        Policy::invalidate();
        rd_step(grid, gpu, Dw, Dg, rho, dt);  // first step: uploads the leaf set
        restore_phi(grid, phi0);
        Policy::invalidate();
        const long up0 = Policy::uploads();
        t0 = now();
        for (int s = 0; s < steps; s++) rd_step(grid, gpu, Dw, Dg, rho, dt);
        t_dropin = now() - t0;
        dropin_uploads = Policy::uploads() - up0;
        FieldMap phi_gpu = snapshot(grid, 0);
        for (int i = 0; i < nb; i++)
            step_mismatch_dropin += count_diff(phi_ref[vInfo[i].blockID], &phi_gpu[vInfo[i].blockID][0], 512);

        restore_phi(grid, phi0);
        Policy::invalidate();
        Policy::deferred_writeback() = true;
        t0 = now();
        for (int s = 0; s < steps; s++) rd_step(grid, gpu, Dw, Dg, rho, dt);
        Policy::sync_host(vInfo, grid.getBlockCollection());
        t_deferred = now() - t0;
        Policy::deferred_writeback() = false;
        FieldMap phi_def = snapshot(grid, 0);
        for (int i = 0; i < nb; i++)
            step_mismatch_deferred += count_diff(phi_ref[vInfo[i].blockID], &phi_def[vInfo[i].blockID][0], 512);

        restore_phi(grid, phi0);
        dev.upload(vInfo, grid.getBlockCollection(), grid.getBoundaryInfo());
        gbfk_mrag::check(dev.ctx, gbfk_rd_step(dev.ctx, Dw, Dg, rho, dt, steps, 1), "gbfk_rd_step");
        std::vector<Real> out((size_t)nb * 512);
        gbfk_mrag::check(dev.ctx, gbfk_download_field(dev.ctx, GBFK_PHI, &out[0], 0, (int64_t)out.size()),
                         "download");
        for (int i = 0; i < nb; i++)
            step_mismatch_resident += count_diff(phi_ref[vInfo[i].blockID], &out[(size_t)i * 512], 512);
        /* faces that are not same-level copies (coarse-fine) */
        const gbfk_mrag::Topology &t = dev.topo;
        for (int i = 0; i < nb; i++) {
            for (int f = 0; f < 6; f++) {
                /* a face is a coarse-fine face if any of its rows is not a single weight-1 entry */
                const int d = f / 2, plus = f % 2;
                bool cf = false;
                int k = 0;
                for (int icode = 0; icode < 27; icode++) {
                    if (icode == 13) continue;
                    const int code[3] = {icode % 3 - 1, (icode / 3) % 3 - 1, (icode / 9) % 3 - 1};
                    int cnt = 1;
                    for (int q = 0; q < 3; q++) cnt *= code[q] == 0 ? 8 : 1;
                    bool is_face = true;
                    for (int q = 0; q < 3; q++)
                        if (q == d ? code[q] != (plus ? 1 : -1) : code[q] != 0) is_face = false;
                    for (int g = 0; g < cnt; g++, k++) {
                        if (!is_face) continue;
                        const int64_t r = (int64_t)i * 488 + k;
                        if (t.row_ptr[r + 1] - t.row_ptr[r] != 1 || t.w0[t.row_ptr[r]] != 1.0) cf = true;
                    }
                }
                n_ghost_faces += cf;
            }
        }
        restore_phi(grid, phi0);
    }

    /* 4. split */
    long split_mismatch = 0;
    int n_split = 0;
    std::set<int> refined_children;
    {
        std::vector<std::pair<double, int> > cand;
        std::vector<FWTReport<1> > rep = BlockFWT<W, B, RD_Projector_Wavelets>::multichannel_fwt<0, 0>(
            vInfo, grid.getBlockCollection(), grid.getBoundaryInfo());
        for (int i = 0; i < nb; i++)
            if (vInfo[i].level < maxLevel) cand.push_back(std::make_pair(-rep[i].getOverAll_DetailMaxMag(), i));
        std::sort(cand.begin(), cand.end());
        std::set<int> want;
        for (size_t k = 0; k < cand.size() && k < 12; k++) want.insert(vInfo[cand[k].second].blockID);

        dev.upload(vInfo, grid.getBlockCollection(), grid.getBoundaryInfo());
        std::map<int, BlockInfo> pre;
        for (int i = 0; i < nb; i++) pre[vInfo[i].blockID] = vInfo[i];
        grid.refine(want);
        grid.getBoundaryInfo();
        std::vector<BlockInfo> post = grid.getBlocksInfo();
        std::set<int> post_ids;
        for (size_t i = 0; i < post.size(); i++) post_ids.insert(post[i].blockID);
        std::vector<int> parents, children;
        std::vector<BlockInfo> parent_info;
        for (int i = 0; i < nb; i++)
            if (!post_ids.count(vInfo[i].blockID)) {
                parents.push_back(i);
                parent_info.push_back(vInfo[i]);
            }
        n_split = (int)parents.size();
        for (int p = 0; p < n_split; p++)
            for (int c = 0; c < 8; c++) children.push_back(nb + 8 * p + c);
        if (n_split > 0)
            gbfk_mrag::check(dev.ctx, gbfk_split(dev.ctx, n_split, &parents[0], &children[0]), "gbfk_split");
        const int fields[3] = {GBFK_PHI, GBFK_PW, GBFK_PG};
        for (int fi = 0; fi < 3; fi++) {
            std::vector<Real> out((size_t)8 * n_split * 512);
            if (n_split)
                gbfk_mrag::check(dev.ctx, gbfk_download_field(dev.ctx, fields[fi], &out[0], (int64_t)nb * 512,
                                                              (int64_t)out.size()),
                                 "download children");
            FieldMap ref = snapshot(grid, fi);
            for (size_t q = 0; q < post.size(); q++) {
                const BlockInfo &ci = post[q];
                for (int p = 0; p < n_split; p++) {
                    const BlockInfo &pi = parent_info[p];
                    if (ci.level != pi.level + 1 || ci.index[0] / 2 != pi.index[0] || ci.index[1] / 2 != pi.index[1] ||
                        ci.index[2] / 2 != pi.index[2])
                        continue;
                    const int c = (ci.index[0] - 2 * pi.index[0]) + 2 * ((ci.index[1] - 2 * pi.index[1]) +
                                                                         2 * (ci.index[2] - 2 * pi.index[2]));
                    split_mismatch += count_diff(ref[ci.blockID], &out[(size_t)(8 * p + c) * 512], 512);
                    if (fi == 0) refined_children.insert(ci.blockID);
                }
            }
        }
    }

    /* 5. collapse: one family of siblings just created */
    long collapse_mismatch = 0;
    int n_collapse = 0;
    {
        std::vector<BlockInfo> cur = grid.getBlocksInfo();
        std::map<std::string, std::vector<int> > fam; /* parent key -> member positions */
        for (size_t i = 0; i < cur.size(); i++) {
            if (!refined_children.count(cur[i].blockID)) continue;
            char key[64];
            snprintf(key, sizeof(key), "%d_%d_%d_%d", cur[i].level, cur[i].index[0] / 2, cur[i].index[1] / 2,
                     cur[i].index[2] / 2);
            fam[key].push_back((int)i);
        }
        std::vector<int> members;
        for (std::map<std::string, std::vector<int> >::iterator it = fam.begin(); it != fam.end(); ++it)
            if (it->second.size() == 8) {
                members = it->second;
                break;
            }
        if (members.size() == 8) {
            dev.upload(cur, grid.getBlockCollection(), grid.getBoundaryInfo());
            std::vector<int> child_slots(8);
            int plevel = cur[members[0]].level - 1, pidx[3] = {cur[members[0]].index[0] / 2,
                                                                 cur[members[0]].index[1] / 2,
                                                                 cur[members[0]].index[2] / 2};
            std::set<int> ids;
            for (int k = 0; k < 8; k++) {
                const BlockInfo &ci = cur[members[k]];
                const int c = (ci.index[0] - 2 * pidx[0]) + 2 * ((ci.index[1] - 2 * pidx[1]) + 2 * (ci.index[2] - 2 * pidx[2]));
                child_slots[c] = members[k];
                ids.insert(ci.blockID);
            }
            const int pslot = (int)cur.size();
            gbfk_mrag::check(dev.ctx, gbfk_collapse(dev.ctx, 1, &child_slots[0], &pslot), "gbfk_collapse");
            int nCollapsed = 0;
            grid.compress(ids, nCollapsed);
            grid.getBoundaryInfo();
            std::vector<BlockInfo> post = grid.getBlocksInfo();
            const int fields[3] = {GBFK_PHI, GBFK_PW, GBFK_PG};
            for (int fi = 0; fi < 3; fi++) {
                std::vector<Real> out(512);
                gbfk_mrag::check(dev.ctx, gbfk_download_field(dev.ctx, fields[fi], &out[0], (int64_t)pslot * 512, 512),
                                 "download parent");
                FieldMap ref = snapshot(grid, fi);
                for (size_t q = 0; q < post.size(); q++)
                    if (post[q].level == plevel && post[q].index[0] == pidx[0] && post[q].index[1] == pidx[1] &&
                        post[q].index[2] == pidx[2]) {
                        collapse_mismatch += count_diff(ref[post[q].blockID], &out[0], 512);
                        if (fi == 0) n_collapse++;
                    }
            }
        }
    }

    printf("{\"real_bytes\": %d, \"blocks\": %d, \"levels\": {", (int)sizeof(Real), nb);
    for (std::map<int, int>::iterator it = levels.begin(); it != levels.end(); ++it)
        printf("%s\"%d\": %d", it == levels.begin() ? "" : ", ", it->first, it->second);
    printf("}, \"coarse_fine_faces\": %d, \"fwt_max\": %.6e, \"fwt_mismatch\": %ld, \"steps\": %d, "
           "\"step_mismatch_dropin\": %ld, \"step_mismatch_deferred\": %ld, \"step_mismatch_resident\": %ld, "
           "\"reference_step_seconds\": %.6f, \"dropin_step_seconds\": %.6f, \"deferred_step_seconds\": %.6f, "
           "\"dropin_uploads\": %ld, \"split_parents\": %d, "
           "\"split_mismatch\": %ld, \"collapsed\": %d, \"collapse_mismatch\": %ld}\n",
           n_ghost_faces, fwt_max, fwt_mismatch, steps, step_mismatch_dropin, step_mismatch_deferred,
           step_mismatch_resident, t_ref, t_dropin, t_deferred, dropin_uploads, n_split, split_mismatch, n_collapse,
           collapse_mismatch);
    return 0;
}
