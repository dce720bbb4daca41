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

#include <pthread.h>
#include <unistd.h>

namespace gbfk_mrag {

template <typename R> struct precision_of;
template <> struct precision_of<double> { static const int value = GBFK_F64; };
template <> struct precision_of<float> { static const int value = GBFK_F32; };

/* Host threads for the per-block loops below: GBFK_HOST_THREADS if set (1 to
 * 64), else the online processors up to 16 (the loops are memory-bound copies
 * and run once per step in the drop-in policy, where thread start-up counts).
 * (The adapter is compiled as C++98 with the reference's sources, hence
 * pthreads.) */
inline int host_threads()
{
    const char *e = getenv("GBFK_HOST_THREADS");
    const long n = e && *e ? atol(e) : std::min(sysconf(_SC_NPROCESSORS_ONLN), 16L);
    return (int)std::max(1L, std::min(n, 64L));
}

template <typename Body> struct RangeTask {
    Body *body;
    size_t begin, end;
    static void *run(void *p)
    {
        RangeTask *t = (RangeTask *)p;
        (*t->body)(t->begin, t->end);
        return NULL;
    }
};

/* body(begin, end) over contiguous ranges covering [0, n), each at least
 * `grain` items, one per thread; the calling thread takes the first range and
 * any range whose thread could not be created.  body must be safe to call
 * concurrently on disjoint ranges. */
template <typename Body>
void parallel_ranges(size_t n, Body &body, size_t grain)
{
    if (n == 0) return;
    grain = std::max<size_t>(grain, 1);
    const size_t nt = std::min((size_t)host_threads(), (n + grain - 1) / grain);
    if (nt <= 1) {
        body(0, n);
        return;
    }
    std::vector<RangeTask<Body> > task(nt);
    std::vector<pthread_t> tid(nt);
    std::vector<char> started(nt, 0);
    for (size_t t = 0; t < nt; t++) {
        task[t].body = &body;
        task[t].begin = n * t / nt;
        task[t].end = n * (t + 1) / nt;
    }
    for (size_t t = 1; t < nt; t++)
        started[t] = pthread_create(&tid[t], NULL, &RangeTask<Body>::run, &task[t]) == 0;
    body(task[0].begin, task[0].end);
    for (size_t t = 1; t < nt; t++) {
        if (started[t]) pthread_join(tid[t], NULL);
        else body(task[t].begin, task[t].end);
    }
}

/* Blocks per thread below which a loop over blocks stays on fewer threads. */
static const size_t kBlocksPerThread = 16;

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

/* The ghost rows of one block: calls row(entries, n) for each of its rows in
 * BlockLab::load order (icode 0..26 without the block itself, 13). */
struct GhostRows {
    static void count(MRAG::BoundaryInfoBlock &bb, int64_t &rows, int64_t &entries)
    {
        const std::vector<std::vector<MRAG::IndexWP> > &ghosts = bb.getGhosts();
        rows = entries = 0;
        for (int icode = 0; icode < 27; icode++) {
            if (icode == 13) continue;
            for (unsigned g = 0; g < bb.boundary[icode].nGhosts; g++) {
                entries += (int64_t)ghosts[bb.boundary[icode].start + g].size();
                rows++;
            }
        }
    }
};

/* Pass 1 of flatten: lock each block's ghost lists and count its rows and
 * entries. */
struct CountGhosts {
    const std::vector<MRAG::BoundaryInfoBlock *> &bbs;
    std::vector<int64_t> &rows, &entries;
    CountGhosts(const std::vector<MRAG::BoundaryInfoBlock *> &b, std::vector<int64_t> &r, std::vector<int64_t> &e)
        : bbs(b), rows(r), entries(e) {}
    void operator()(size_t begin, size_t end) const
    {
        for (size_t i = begin; i < end; i++) {
            bbs[i]->lock();
            GhostRows::count(*bbs[i], rows[i], entries[i]);
        }
    }
};

/* Pass 2: write each block's rows at its offsets, then release its lists. */
template <typename BlockInfoT>
struct FillGhosts {
    const std::vector<BlockInfoT> &vInfo;
    const std::vector<MRAG::BoundaryInfoBlock *> &bbs;
    const std::vector<int64_t> &row_off, &entry_off;
    Topology &t;
    int max_id;
    FillGhosts(const std::vector<BlockInfoT> &v, const std::vector<MRAG::BoundaryInfoBlock *> &b,
               const std::vector<int64_t> &ro, const std::vector<int64_t> &eo, Topology &top, int mx)
        : vInfo(v), bbs(b), row_off(ro), entry_off(eo), t(top), max_id(mx) {}
    void operator()(size_t begin, size_t end) const
    {
        for (size_t i = begin; i < end; i++) {
            MRAG::BoundaryInfoBlock &bb = *bbs[i];
            const std::vector<std::vector<MRAG::IndexWP> > &ghosts = bb.getGhosts();
            const std::vector<MRAG::PointIndex> &pool = bb.getIndexPool();
            int64_t r = row_off[i], k = entry_off[i];
            for (int icode = 0; icode < 27; icode++) {
                if (icode == 13) continue;
                for (unsigned g = 0; g < bb.boundary[icode].nGhosts; g++) {
                    const std::vector<MRAG::IndexWP> &row = ghosts[bb.boundary[icode].start + g];
                    for (size_t q = 0; q < row.size(); q++, k++) {
                        const MRAG::PointIndex &p = pool[row[q].point_index];
                        const int slot = p.blockID >= 0 && p.blockID <= max_id ? t.slot_of[p.blockID] : -1;
                        if (slot < 0) {
                            fprintf(stderr, "gbfk_mrag: a ghost of block %d reads block %d, not a leaf\n",
                                    vInfo[i].blockID, p.blockID);
                            abort();
                        }
                        t.src[k] = (int64_t)slot * GBFK_BLOCK_CELLS + p.index;
                        t.w0[k] = bb.weightsPool[row[q].weights_index[0]];
                        t.w1[k] = bb.weightsPool[row[q].weights_index[1]];
                        t.w2[k] = bb.weightsPool[row[q].weights_index[2]];
                    }
                    t.row_ptr[++r] = k;
                }
            }
            bb.release();
        }
    }
};

/* The leaves of vInfo (slot = position) and their ghost lists, flattened
 * into t in two parallel passes over the blocks (count, then fill at prefix
 * offsets); the result does not depend on the number of threads.  t's
 * vectors are reused, so a caller that keeps t across topology changes
 * allocates only when the lists grow. */
template <typename BlockInfoT, typename BoundaryInfoT>
void flatten_into(Topology &t, const std::vector<BlockInfoT> &vInfo, BoundaryInfoT &boundaryInfo)
{
    const size_t nb = vInfo.size();
    int max_id = -1;
    for (size_t i = 0; i < nb; i++) max_id = std::max(max_id, vInfo[i].blockID);
    t.slot_of.assign((size_t)(max_id + 1), -1);
    t.blocks.clear();
    t.blocks.reserve(nb);
    std::vector<MRAG::BoundaryInfoBlock *> bbs(nb);
    for (size_t i = 0; i < nb; i++) {
        gbfk_blockinfo b;
        b.slot = (int)i;
        b.level = vInfo[i].level;
        b.index[0] = vInfo[i].index[0];
        b.index[1] = vInfo[i].index[1];
        b.index[2] = vInfo[i].index[2];
        b.h = (double)vInfo[i].h[0];
        t.blocks.push_back(b);
        t.slot_of[vInfo[i].blockID] = (int)i;
        typename std::map<int, MRAG::BoundaryInfoBlock *>::iterator it =
            boundaryInfo.boundaryInfoOfBlock.find(vInfo[i].blockID);
        if (it == boundaryInfo.boundaryInfoOfBlock.end()) {
            fprintf(stderr, "gbfk_mrag: block %d has no ghost lists\n", vInfo[i].blockID);
            abort();
        }
        bbs[i] = it->second;
    }
    std::vector<int64_t> rows(nb), entries(nb), row_off(nb + 1, 0), entry_off(nb + 1, 0);
    CountGhosts count(bbs, rows, entries);
    parallel_ranges(nb, count, kBlocksPerThread);
    for (size_t i = 0; i < nb; i++) {
        row_off[i + 1] = row_off[i] + rows[i];
        entry_off[i + 1] = entry_off[i] + entries[i];
    }
    t.row_ptr.resize((size_t)row_off[nb] + 1);
    t.row_ptr[0] = 0;
    t.src.resize((size_t)entry_off[nb]);
    t.w0.resize(t.src.size());
    t.w1.resize(t.src.size());
    t.w2.resize(t.src.size());
    FillGhosts<BlockInfoT> fill(vInfo, bbs, row_off, entry_off, t, max_id);
    parallel_ranges(nb, fill, kBlocksPerThread);
}

template <typename BlockInfoT, typename BoundaryInfoT>
Topology flatten(const std::vector<BlockInfoT> &vInfo, BoundaryInfoT &boundaryInfo)
{
    Topology t;
    flatten_into(t, vInfo, boundaryInfo);
    return t;
}

/* One Cell field of every block, slot-major (512 Reals per block), and back;
 * blocks in parallel. */
template <typename R, typename Collection, typename BlockInfoT, typename Field>
struct GatherBody {
    R *out;
    const Collection &c;
    const std::vector<BlockInfoT> &vInfo;
    Field field;
    GatherBody(R *o, const Collection &col, const std::vector<BlockInfoT> &v, Field f)
        : out(o), c(col), vInfo(v), field(f) {}
    void operator()(size_t begin, size_t end) const
    {
        typedef typename Collection::BlockType B;
        for (size_t i = begin; i < end; i++) {
            B &block = c[vInfo[i].blockID];
            R *o = out + i * GBFK_BLOCK_CELLS;
            for (int iz = 0; iz < B::sizeZ; iz++)
                for (int iy = 0; iy < B::sizeY; iy++)
                    for (int ix = 0; ix < B::sizeX; ix++) *o++ = field(block(ix, iy, iz));
        }
    }
};

template <typename R, typename Collection, typename BlockInfoT, typename Field>
void gather_into(std::vector<R> &out, const Collection &c, const std::vector<BlockInfoT> &vInfo, Field field)
{
    out.resize(vInfo.size() * GBFK_BLOCK_CELLS);
    if (vInfo.empty()) return;
    GatherBody<R, Collection, BlockInfoT, Field> body(&out[0], c, vInfo, field);
    parallel_ranges(vInfo.size(), body, kBlocksPerThread);
}

template <typename R, typename Collection, typename BlockInfoT, typename Setter>
struct ScatterBody {
    const R *in;
    const Collection &c;
    const std::vector<BlockInfoT> &vInfo;
    Setter set;
    ScatterBody(const R *p, const Collection &col, const std::vector<BlockInfoT> &v, Setter s)
        : in(p), c(col), vInfo(v), set(s) {}
    void operator()(size_t begin, size_t end) const
    {
        typedef typename Collection::BlockType B;
        for (size_t i = begin; i < end; i++) {
            B &block = c[vInfo[i].blockID];
            const R *p = in + i * GBFK_BLOCK_CELLS;
            for (int iz = 0; iz < B::sizeZ; iz++)
                for (int iy = 0; iy < B::sizeY; iy++)
                    for (int ix = 0; ix < B::sizeX; ix++) set(block(ix, iy, iz), *p++);
        }
    }
};

template <typename R, typename Collection, typename BlockInfoT, typename Setter>
void scatter_from(const std::vector<R> &in, const Collection &c, const std::vector<BlockInfoT> &vInfo, Setter set)
{
    if (vInfo.empty()) return;
    ScatterBody<R, Collection, BlockInfoT, Setter> body(&in[0], c, vInfo, set);
    parallel_ranges(vInfo.size(), body, kBlocksPerThread);
}

/* p_w, p_g and phi of every block in one pass over the Cells. */
template <typename R, typename Collection, typename BlockInfoT>
struct GatherAnatomyBody {
    R *pw, *pg, *phi;
    const Collection &c;
    const std::vector<BlockInfoT> &vInfo;
    GatherAnatomyBody(R *a, R *b, R *f, const Collection &col, const std::vector<BlockInfoT> &v)
        : pw(a), pg(b), phi(f), c(col), vInfo(v) {}
    void operator()(size_t begin, size_t end) const
    {
        typedef typename Collection::BlockType B;
        for (size_t i = begin; i < end; i++) {
            B &block = c[vInfo[i].blockID];
            size_t o = i * GBFK_BLOCK_CELLS;
            for (int iz = 0; iz < B::sizeZ; iz++)
                for (int iy = 0; iy < B::sizeY; iy++)
                    for (int ix = 0; ix < B::sizeX; ix++, o++) {
                        const typename B::ElementType &cell = block(ix, iy, iz);
                        pw[o] = cell.p_w;
                        pg[o] = cell.p_g;
                        phi[o] = cell.phi;
                    }
        }
    }
};

template <typename R, typename Collection, typename BlockInfoT>
void gather_anatomy(std::vector<R> &pw, std::vector<R> &pg, std::vector<R> &phi, const Collection &c,
                    const std::vector<BlockInfoT> &vInfo)
{
    const size_t n = vInfo.size() * GBFK_BLOCK_CELLS;
    pw.resize(n);
    pg.resize(n);
    phi.resize(n);
    if (vInfo.empty()) return;
    GatherAnatomyBody<R, Collection, BlockInfoT> body(&pw[0], &pg[0], &phi[0], c, vInfo);
    parallel_ranges(vInfo.size(), body, kBlocksPerThread);
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
        flatten_into(topo, vInfo, b);
        const gbfk_ghost_csr csr = topo.csr();
        check(ctx, gbfk_set_topology(ctx, &topo.blocks[0], (int)topo.blocks.size(), &csr), "gbfk_set_topology");
        ids.clear();
        for (size_t i = 0; i < vInfo.size(); i++) ids.push_back(vInfo[i].blockID);
        std::vector<Real> pw, pg, phi;
        gather_anatomy(pw, pg, phi, c, vInfo);
        check(ctx, gbfk_upload_field(ctx, GBFK_PW, &pw[0], 0, (int64_t)pw.size()), "upload p_w");
        check(ctx, gbfk_upload_field(ctx, GBFK_PG, &pg[0], 0, (int64_t)pg.size()), "upload p_g");
        check(ctx, gbfk_upload_field(ctx, GBFK_PHI, &phi[0], 0, (int64_t)phi.size()), "upload phi");
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
