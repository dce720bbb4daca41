/*
 * gbfk_mrag.hpp -- C++ adapter from MRAG (the reference's grid library) to the
 * gbfk C ABI.  Header-only; include it after the reference's headers
 * (Glioma/Glioma_Types.h), link libgbfk.so.
 *
 * Two levels of use:
 *  1. The drop-in policy BlockProcessing_CUDA<B>: the typedef in
 *     Glioma/Glioma_Types.h:306-312 becomes
 *         typedef gbfk_mrag::BlockProcessing_CUDA<B> BlockProcessing;
 *     and Glioma_ReactionDiffusion::_reactionDiffusionStep
 *     (Glioma/Glioma_ReactionDiffusion.cpp:176-187) runs unchanged: its
 *     pipeline_process(..., ReactionDiffusionOperator) records Dw, Dg, rho and
 *     the following process(..., UpdateTumor) launches one fused step on the
 *     GPU.  The blocks stay authoritative on the host: each step uploads phi
 *     (and, after a topology or anatomy change, p_w, p_g and the ghost lists)
 *     and writes phi back into the Cells.
 *  2. The building blocks below (upload_topology, gather/scatter of Cell
 *     fields) for a driver that keeps the data on the GPU across many steps
 *     and only reads it back for dumps and refinement.
 *
 * Blocks of a topology live in pool slot = their position in vInfo.
 */
#pragma once
#include "gbfk.h"

#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <map>
#include <vector>

namespace gbfk_mrag {

template <typename R> struct precision_of;
template <> struct precision_of<double> { static const int value = GBFK_F64; };
template <> struct precision_of<float> { static const int value = GBFK_F32; };

/* Leaf blocks and ghost lists of a grid in the layout of gbfk_ghost_csr
 * (include/gbfk.h): blocks in vInfo order, ghosts in BlockLab::load order
 * (MRAG/MRAGcore/MRAGBlockLab.h:256-279). */
struct Topology {
    std::vector<gbfk_blockinfo> blocks;
    std::vector<int> slot_of; /* blockID -> slot (-1: not a leaf) */
    std::vector<int64_t> row_ptr, src;
    std::vector<double> w0, w1, w2;
    gbfk_ghost_csr csr() const
    {
        gbfk_ghost_csr c;
        c.nrows = (int64_t)row_ptr.size() - 1;
        c.row_ptr = &row_ptr[0];
        c.src = src.empty() ? NULL : &src[0];
        c.w0 = w0.empty() ? NULL : &w0[0];
        c.w1 = w1.empty() ? NULL : &w1[0];
        c.w2 = w2.empty() ? NULL : &w2[0];
        return c;
    }
};

template <typename BlockInfoT, typename BoundaryInfoT>
Topology flatten(const std::vector<BlockInfoT> &vInfo, BoundaryInfoT &boundaryInfo)
{
    Topology t;
    int max_id = -1;
    for (size_t i = 0; i < vInfo.size(); i++) max_id = std::max(max_id, vInfo[i].blockID);
    t.slot_of.assign((size_t)(max_id + 1), -1);
    t.blocks.reserve(vInfo.size());
    t.row_ptr.reserve(vInfo.size() * GBFK_LAB_GHOSTS + 1);
    t.src.reserve(vInfo.size() * GBFK_LAB_GHOSTS * 2);
    t.w0.reserve(t.src.capacity());
    t.w1.reserve(t.src.capacity());
    t.w2.reserve(t.src.capacity());
    for (int i = 0; i < (int)vInfo.size(); i++) {
        gbfk_blockinfo b;
        b.slot = i;
        b.level = vInfo[i].level;
        b.index[0] = vInfo[i].index[0];
        b.index[1] = vInfo[i].index[1];
        b.index[2] = vInfo[i].index[2];
        b.h = (double)vInfo[i].h[0];
        t.blocks.push_back(b);
        t.slot_of[vInfo[i].blockID] = i;
    }
    t.row_ptr.push_back(0);
    for (size_t i = 0; i < vInfo.size(); i++) {
        typename std::map<int, MRAG::BoundaryInfoBlock *>::iterator it =
            boundaryInfo.boundaryInfoOfBlock.find(vInfo[i].blockID);
        if (it == boundaryInfo.boundaryInfoOfBlock.end()) {
            fprintf(stderr, "gbfk_mrag: block %d has no ghost lists\n", vInfo[i].blockID);
            abort();
        }
        MRAG::BoundaryInfoBlock &bb = *it->second;
        bb.lock();
        const std::vector<std::vector<MRAG::IndexWP> > &ghosts = bb.getGhosts();
        const std::vector<MRAG::PointIndex> &pool = bb.getIndexPool();
        for (int icode = 0; icode < 27; icode++) {
            if (icode == 13) continue;
            for (unsigned g = 0; g < bb.boundary[icode].nGhosts; g++) {
                const std::vector<MRAG::IndexWP> &row = ghosts[bb.boundary[icode].start + g];
                for (size_t k = 0; k < row.size(); k++) {
                    const MRAG::PointIndex &p = pool[row[k].point_index];
                    const int slot = p.blockID >= 0 && p.blockID <= max_id ? t.slot_of[p.blockID] : -1;
                    if (slot < 0) {
                        fprintf(stderr, "gbfk_mrag: a ghost of block %d reads block %d, not a leaf\n",
                                vInfo[i].blockID, p.blockID);
                        abort();
                    }
                    t.src.push_back((int64_t)slot * GBFK_BLOCK_CELLS + p.index);
                    t.w0.push_back(bb.weightsPool[row[k].weights_index[0]]);
                    t.w1.push_back(bb.weightsPool[row[k].weights_index[1]]);
                    t.w2.push_back(bb.weightsPool[row[k].weights_index[2]]);
                }
                t.row_ptr.push_back((int64_t)t.src.size());
            }
        }
        bb.release();
    }
    return t;
}

/* One Cell field of every block, slot-major (512 Reals per block), and back. */
template <typename R, typename Collection, typename BlockInfoT, typename Field>
void gather_into(std::vector<R> &out, const Collection &c, const std::vector<BlockInfoT> &vInfo, Field field)
{
    typedef typename Collection::BlockType B;
    out.resize(vInfo.size() * GBFK_BLOCK_CELLS);
    for (size_t i = 0; i < vInfo.size(); i++) {
        B &block = c[vInfo[i].blockID];
        R *o = &out[i * GBFK_BLOCK_CELLS];
        for (int iz = 0; iz < B::sizeZ; iz++)
            for (int iy = 0; iy < B::sizeY; iy++)
                for (int ix = 0; ix < B::sizeX; ix++) *o++ = field(block(ix, iy, iz));
    }
}

template <typename R, typename Collection, typename BlockInfoT, typename Setter>
void scatter_from(const std::vector<R> &in, const Collection &c, const std::vector<BlockInfoT> &vInfo, Setter set)
{
    typedef typename Collection::BlockType B;
    for (size_t i = 0; i < vInfo.size(); i++) {
        B &block = c[vInfo[i].blockID];
        const R *p = &in[i * GBFK_BLOCK_CELLS];
        for (int iz = 0; iz < B::sizeZ; iz++)
            for (int iy = 0; iy < B::sizeY; iy++)
                for (int ix = 0; ix < B::sizeX; ix++) set(block(ix, iy, iz), *p++);
    }
}

template <typename Cell> struct get_phi { Real operator()(const Cell &c) const { return c.phi; } };
template <typename Cell> struct get_pw { Real operator()(const Cell &c) const { return c.p_w; } };
template <typename Cell> struct get_pg { Real operator()(const Cell &c) const { return c.p_g; } };
template <typename Cell> struct set_phi { void operator()(Cell &c, Real v) const { c.phi = v; } };
template <typename Cell> struct set_pw { void operator()(Cell &c, Real v) const { c.p_w = v; } };
template <typename Cell> struct set_pg { void operator()(Cell &c, Real v) const { c.p_g = v; } };

inline void check(gbfk_ctx *ctx, int rc, const char *what)
{
    if (rc != GBFK_OK) {
        fprintf(stderr, "gbfk_mrag: %s failed (%d): %s\n", what, rc, ctx ? gbfk_last_error(ctx) : "");
        abort();
    }
}

/* A gbfk context holding one MRAG grid's leaf set. */
class Device {
public:
    gbfk_ctx *ctx;
    Topology topo;
    std::vector<int> ids; /* blockIDs of the uploaded topology, in vInfo order */

    explicit Device(int max_blocks, int device = 0) : ctx(NULL)
    {
        gbfk_config cfg;
        cfg.precision = precision_of<Real>::value;
        cfg.max_blocks = max_blocks;
        cfg.device = device;
        cfg.stream = NULL;
        check(NULL, gbfk_create(&cfg, &ctx), "gbfk_create");
    }
    ~Device() { gbfk_destroy(ctx); }

    bool same_leaves(const std::vector<MRAG::BlockInfo> &vInfo) const
    {
        if (vInfo.size() != ids.size()) return false;
        for (size_t i = 0; i < vInfo.size(); i++)
            if (vInfo[i].blockID != ids[i]) return false;
        return true;
    }

    /* Upload leaves, ghost lists and the three fields. */
    template <typename Collection>
    void upload(const std::vector<MRAG::BlockInfo> &vInfo, const Collection &c, MRAG::BoundaryInfo &b)
    {
        typedef typename Collection::BlockType::ElementType Cell;
        topo = flatten(vInfo, b);
        const gbfk_ghost_csr csr = topo.csr();
        check(ctx, gbfk_set_topology(ctx, &topo.blocks[0], (int)topo.blocks.size(), &csr), "gbfk_set_topology");
        ids.clear();
        for (size_t i = 0; i < vInfo.size(); i++) ids.push_back(vInfo[i].blockID);
        std::vector<Real> f;
        gather_into(f, c, vInfo, get_pw<Cell>());
        check(ctx, gbfk_upload_field(ctx, GBFK_PW, &f[0], 0, (int64_t)f.size()), "upload p_w");
        gather_into(f, c, vInfo, get_pg<Cell>());
        check(ctx, gbfk_upload_field(ctx, GBFK_PG, &f[0], 0, (int64_t)f.size()), "upload p_g");
        upload_phi(vInfo, c);
    }

    template <typename Collection>
    void upload_phi(const std::vector<MRAG::BlockInfo> &vInfo, const Collection &c)
    {
        typedef typename Collection::BlockType::ElementType Cell;
        std::vector<Real> f;
        gather_into(f, c, vInfo, get_phi<Cell>());
        check(ctx, gbfk_upload_field(ctx, GBFK_PHI, &f[0], 0, (int64_t)f.size()), "upload phi");
    }

    template <typename Collection>
    void download_phi(const std::vector<MRAG::BlockInfo> &vInfo, const Collection &c)
    {
        typedef typename Collection::BlockType::ElementType Cell;
        std::vector<Real> f(vInfo.size() * GBFK_BLOCK_CELLS);
        check(ctx, gbfk_download_field(ctx, GBFK_PHI, &f[0], 0, (int64_t)f.size()), "download phi");
        scatter_from(f, c, vInfo, set_phi<Cell>());
    }
};

/* The drop-in BlockProcessing policy for the RD step (see the file comment). */
template <typename BlockType>
class BlockProcessing_CUDA {
    struct Pending {
        bool set;
        Real Dw, Dg, rho;
        const void *collection;
        MRAG::BoundaryInfo *boundaryInfo;
        Pending() : set(false), Dw(0), Dg(0), rho(0), collection(NULL), boundaryInfo(NULL) {}
    };
    static Pending &pending()
    {
        static Pending p;
        return p;
    }
    static Device *&device()
    {
        static Device *d = NULL;
        return d;
    }

public:
    /* Capacity of the device pool in blocks (set before the first step). */
    static int &max_blocks()
    {
        static int n = 1 << 16;
        return n;
    }
    /* Drop the cached topology (after refine/compress or a new anatomy). */
    static void invalidate()
    {
        if (device()) device()->ids.clear();
    }

    /* MRAGBlockProcessing_TBB.h:476 -- records the operator's coefficients. */
    template <typename Processing, typename Collection>
    void pipeline_process(std::vector<MRAG::BlockInfo> &vInfo, Collection &c, MRAG::BoundaryInfo &b,
                          Processing &p)
    {
        (void)vInfo;
        Pending &q = pending();
        q.set = true;
        q.Dw = p.Dw;
        q.Dg = p.Dg;
        q.rho = p.rho;
        q.collection = &c;
        q.boundaryInfo = &b;
    }

    /* MRAGBlockProcessing_TBB.h:249 -- the UpdateTumor sweep: runs the fused
     * step and writes phi back into the Cells. */
    template <typename Processing, typename Collection>
    static void process(std::vector<MRAG::BlockInfo> &vInfo, Collection &c, Processing &p, int nGranularity = -1)
    {
        (void)nGranularity;
        Pending &q = pending();
        if (!q.set || q.collection != (const void *)&c) {
            fprintf(stderr, "gbfk_mrag: UpdateTumor without a preceding ReactionDiffusionOperator sweep\n");
            abort();
        }
        q.set = false;
        if (!device()) device() = new Device(max_blocks());
        Device &d = *device();
        if (!d.same_leaves(vInfo)) d.upload(vInfo, c, *q.boundaryInfo);
        else d.upload_phi(vInfo, c);
        check(d.ctx, gbfk_rd_step(d.ctx, q.Dw, q.Dg, q.rho, p.dt, 1, 0), "gbfk_rd_step");
        d.download_phi(vInfo, c);
    }
};

}  // namespace gbfk_mrag
