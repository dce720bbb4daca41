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
 *     GPU.  phi stays on the device between topology changes (the leaf set,
 *     its ghost lists, p_w, p_g and phi are uploaded after a refine or
 *     compress) and is written back into the Cells after each step, or only
 *     at sync_host() with deferred_writeback().
 *  2. Resident adaptivity (ResidentGrid, DeviceSplitter, DeviceCollapser,
 *     AutomaticRefinement, AutomaticCompression below): the leaves stay in GPU
 *     memory for the whole run, including re-adaptation; the grid keeps only
 *     the block tree (dropin/glioma_adaptive.cpp).
 *  3. The building blocks (flatten of the ghost lists, gather/scatter of Cell
 *     fields) for other drivers.
 *
 * Blocks of a topology live in pool slot = their position in vInfo (levels 1
 * and 3) or keep one slot for their lifetime (ResidentGrid).  Failures raise
 * gbfk_mrag::Error.
 */
#pragma once
#include "gbfk.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <algorithm>
#include <map>
#include <set>
#include <stdexcept>
#include <string>
#include <vector>

#include <pthread.h>
#include <sys/time.h>
#include <unistd.h>

namespace gbfk_mrag {

/* Raised by the adapter on a failed library call or an inconsistent grid:
 * the reference's interfaces return void, so errors travel as exceptions
 * (code = the gbfk status) instead of aborting the process. */
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

inline void ok(gbfk_ctx *ctx, int rc, const char *what)
{
    if (rc != GBFK_OK)
        throw Error(rc, std::string(what) + ": " + (ctx ? gbfk_last_error(ctx) : "no context"));
}

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
                            char m[128];
                            snprintf(m, sizeof m, "gbfk_mrag: a ghost of block %d reads block %d, not a leaf",
                                     vInfo[i].blockID, p.blockID);
                            throw Error(GBFK_E_INVALID, m);
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

/* The leaves of vInfo and their ghost lists, flattened into t in two
 * parallel passes over the blocks (count, then fill at prefix offsets); the
 * result does not depend on the number of threads.  Block i lives in slot
 * slots[i], or in slot i when slots is NULL.  t's vectors are reused, so a
 * caller that keeps t across topology changes allocates only when the lists
 * grow. */
template <typename BlockInfoT, typename BoundaryInfoT>
void flatten_into(Topology &t, const std::vector<BlockInfoT> &vInfo, BoundaryInfoT &boundaryInfo,
                  const std::vector<int> *slots = NULL)
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
        b.slot = slots ? (*slots)[i] : (int)i;
        b.level = vInfo[i].level;
        b.index[0] = vInfo[i].index[0];
        b.index[1] = vInfo[i].index[1];
        b.index[2] = vInfo[i].index[2];
        b.h = (double)vInfo[i].h[0];
        t.blocks.push_back(b);
        t.slot_of[vInfo[i].blockID] = b.slot;
        typename std::map<int, MRAG::BoundaryInfoBlock *>::iterator it =
            boundaryInfo.boundaryInfoOfBlock.find(vInfo[i].blockID);
        if (it == boundaryInfo.boundaryInfoOfBlock.end()) {
            char m[96];
            snprintf(m, sizeof m, "gbfk_mrag: block %d has no ghost lists", vInfo[i].blockID);
            throw Error(GBFK_E_STATE, m);
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

/* A failed call raises Error (see ok). */
inline void check(gbfk_ctx *ctx, int rc, const char *what) { ok(ctx, rc, what); }

/* phi of every block from a slot-major buffer (the Cell type from the collection). */
template <typename R, typename Collection, typename BlockInfoT>
void scatter_phi(const std::vector<R> &in, const Collection &c, const std::vector<BlockInfoT> &vInfo)
{
    typedef typename Collection::BlockType::ElementType Cell;
    scatter_from(in, c, vInfo, set_phi<Cell>());
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

/* The drop-in BlockProcessing policy for the RD step (see the file comment).
 *
 * The device copy of phi is authoritative between topology changes: the
 * leaves, their ghost lists, p_w, p_g and phi are uploaded when the leaf set
 * differs from the device's (after refine / compress), and otherwise the step
 * runs on the device state without an upload.  After each step phi is written
 * back into the Cells, so that the driver's dumps and its host refinement see
 * the current state; with deferred_writeback() set, the write-back waits for
 * sync_host(), which the caller makes before it reads the Cells.  A caller
 * that changes phi, p_w or p_g in the Cells without changing the leaf set
 * calls invalidate() (or sets verify_mirror(), which compares the Cells' phi
 * with the device's last state before every step and re-uploads on a
 * difference, at the cost of reading the Cells each step).  Errors raise
 * gbfk_mrag::Error. */
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
    /* phi as last written back (for verify_mirror) and whether the Cells are behind the device */
    static std::vector<Real> &mirror()
    {
        static std::vector<Real> m;
        return m;
    }
    static bool &host_stale()
    {
        static bool b = false;
        return b;
    }

public:
    /* Capacity of the device pool in blocks (set before the first step). */
    static int &max_blocks()
    {
        static int n = 1 << 16;
        return n;
    }
    static bool &deferred_writeback()
    {
        static bool b = false;
        return b;
    }
    static bool &verify_mirror()
    {
        static bool b = false;
        return b;
    }
    /* Steps, uploads of the whole leaf set and write-backs so far. */
    static long &steps()
    {
        static long n = 0;
        return n;
    }
    static long &uploads()
    {
        static long n = 0;
        return n;
    }
    static long &writebacks()
    {
        static long n = 0;
        return n;
    }
    /* Drop the device's copy (after changing phi, p_w or p_g in the Cells by hand). */
    static void invalidate()
    {
        if (device()) device()->ids.clear();
    }
    /* Write phi back into the Cells if the device is ahead of them. */
    template <typename Collection>
    static void sync_host(const std::vector<MRAG::BlockInfo> &vInfo, const Collection &c)
    {
        if (!host_stale() || !device()) return;
        Device &d = *device();
        if (!d.same_leaves(vInfo)) throw Error(GBFK_E_STATE, "sync_host: the leaf set changed since the last step");
        write_back(d, vInfo, c);
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

    /* MRAGBlockProcessing_TBB.h:249 -- the UpdateTumor sweep: one fused step on
     * the device (see the class comment for when phi moves). */
    template <typename Processing, typename Collection>
    static void process(std::vector<MRAG::BlockInfo> &vInfo, Collection &c, Processing &p, int nGranularity = -1)
    {
        typedef typename Collection::BlockType::ElementType Cell;
        (void)nGranularity;
        Pending &q = pending();
        if (!q.set || q.collection != (const void *)&c)
            throw Error(GBFK_E_STATE, "gbfk_mrag: UpdateTumor without a preceding ReactionDiffusionOperator sweep");
        q.set = false;
        if (!device()) device() = new Device(max_blocks());
        Device &d = *device();
        if (!d.same_leaves(vInfo)) {
            if (host_stale()) throw Error(GBFK_E_STATE, "gbfk_mrag: the leaf set changed while phi was only on the "
                                                        "device (call sync_host before refining)");
            d.upload(vInfo, c, *q.boundaryInfo);
            uploads()++;
            mirror().clear();
        } else if (verify_mirror()) {
            std::vector<Real> f;
            gather_into(f, c, vInfo, get_phi<Cell>());
            if (host_stale() || f.size() != mirror().size() ||
                memcmp(&f[0], &mirror()[0], f.size() * sizeof(Real)) != 0) {
                check(d.ctx, gbfk_upload_field(d.ctx, GBFK_PHI, &f[0], 0, (int64_t)f.size()), "upload phi");
                host_stale() = false;
            }
        }
        check(d.ctx, gbfk_rd_step(d.ctx, q.Dw, q.Dg, q.rho, p.dt, 1, 0), "gbfk_rd_step");
        steps()++;
        host_stale() = true;
        if (!deferred_writeback()) write_back(d, vInfo, c);
    }

private:
    template <typename Collection>
    static void write_back(Device &d, const std::vector<MRAG::BlockInfo> &vInfo, const Collection &c)
    {
        typedef typename Collection::BlockType::ElementType Cell;
        std::vector<Real> &f = mirror();
        f.resize(vInfo.size() * GBFK_BLOCK_CELLS);
        check(d.ctx, gbfk_download_field(d.ctx, GBFK_PHI, &f[0], 0, (int64_t)f.size()), "download phi");
        scatter_from(f, c, vInfo, set_phi<Cell>());
        host_stale() = false;
        writebacks()++;
    }
};


/* ---------------------------------------------------------------------------
 * Resident adaptivity: the leaves live in the device pool for the whole run;
 * the caller's MRAG grid keeps only the block tree.
 *
 * The reference adapts with Science::AutomaticRefinement / AutomaticCompression
 * (MRAG/MRAGscience/MRAGScienceCore.h:42-177): per block the wavelet detail of
 * phi (BlockFWT::multichannel_fwt), then Grid::refine / Grid::compress, whose
 * plans (Refiner::createPlan, Compressor::createPlan) are realised by the
 * grid's BlockSplitter and BlockCollapser on host Cells
 * (MRAG/MRAGcore/MRAGrid.inl:248-350,384-470).  Here the details come from the
 * device (gbfk_fwt_details), the grid still makes its own plans, and the
 * splitter and collapser the grid calls are DeviceSplitter / DeviceCollapser:
 * they create and erase the grid's block IDs exactly as the reference's do
 * (so the tree and its IDs evolve identically) but move the data with
 * gbfk_split / gbfk_collapse on the device.  Blocks keep their pool slot for
 * as long as they exist, so a topology change moves no data; only the new
 * ghost lists are uploaded.  The host Cells of the grid are not kept current
 * (download_phi writes phi back for a dump).
 * ------------------------------------------------------------------------- */


inline double wall_seconds()
{
    timeval tv;
    gettimeofday(&tv, NULL);
    return tv.tv_sec + 1e-6 * tv.tv_usec;
}

/* Pool slots by block ID: a free list over [0, capacity). */
class SlotMap {
    std::map<int, int> slot_;
    std::vector<int> free_;

public:
    explicit SlotMap(int capacity = 0) { reset(capacity); }
    void reset(int capacity)
    {
        slot_.clear();
        free_.clear();
        for (int s = capacity - 1; s >= 0; s--) free_.push_back(s);
    }
    int acquire(int id)
    {
        if (slot_.count(id)) throw Error(GBFK_E_INVALID, "SlotMap: block already has a slot");
        if (free_.empty()) throw Error(GBFK_E_OOM, "SlotMap: the device pool is full");
        const int s = free_.back();
        free_.pop_back();
        slot_[id] = s;
        return s;
    }
    void release(int id)
    {
        std::map<int, int>::iterator it = slot_.find(id);
        if (it == slot_.end()) throw Error(GBFK_E_INVALID, "SlotMap: block has no slot");
        free_.push_back(it->second);
        slot_.erase(it);
    }
    int slot(int id) const
    {
        std::map<int, int>::const_iterator it = slot_.find(id);
        if (it == slot_.end()) throw Error(GBFK_E_INVALID, "SlotMap: block has no slot");
        return it->second;
    }
    size_t size() const { return slot_.size(); }
};

/* A detail within `rel` (relative) of the tolerance it was compared with:
 * a decision that rounding of the state could flip. */
struct NearDecision {
    int adaptation, level, index[3];
    double detail, tol;
};

/* Timings and counters of a resident run (host wall seconds; the device calls
 * inside them synchronise). */
struct ResidentStats {
    int uploads, splits, collapses, detail_sweeps;
    double t_upload, t_details, t_plan, t_split, t_collapse;
    ResidentStats()
        : uploads(0), splits(0), collapses(0), detail_sweeps(0), t_upload(0), t_details(0), t_plan(0), t_split(0),
          t_collapse(0) {}
};

/* The device side of an MRAG grid whose leaves stay in GPU memory. */
template <typename GridT>
class ResidentGrid {
public:
    gbfk_ctx *ctx;
    SlotMap slots;
    std::vector<int> ids; /* block IDs of the uploaded topology, in upload order */
    std::map<int, int> pos_of; /* block ID -> position in the uploaded topology */
    Topology topo;
    ResidentStats stats;
    int adaptation;                  /* counter for NearDecision records */
    double near_rel;                 /* what counts as near a tolerance */
    std::vector<NearDecision> near;  /* decisions within near_rel of their tolerance */
    double min_margin_refine, min_margin_compress; /* smallest |detail/tol - 1| seen */

    ResidentGrid(int capacity, int device = 0)
        : ctx(NULL), slots(capacity), adaptation(0), near_rel(1e-6), min_margin_refine(HUGE_VAL),
          min_margin_compress(HUGE_VAL), capacity_(capacity)
    {
        gbfk_config cfg;
        cfg.precision = precision_of<Real>::value;
        cfg.max_blocks = capacity;
        cfg.device = device;
        cfg.stream = NULL;
        ok(NULL, gbfk_create(&cfg, &ctx), "gbfk_create");
    }
    ~ResidentGrid() { gbfk_destroy(ctx); }

    /* Every leaf gets a slot; topology, p_w, p_g and phi are uploaded from the
     * grid's Cells (once, before the time loop). */
    void upload_all(GridT &g)
    {
        std::vector<MRAG::BlockInfo> vInfo = g.getBlocksInfo();
        slots.reset(capacity_);
        for (size_t i = 0; i < vInfo.size(); i++) slots.acquire(vInfo[i].blockID);
        upload_topology(g, vInfo);
        std::vector<Real> pw, pg, phi;
        gather_anatomy(pw, pg, phi, g.getBlockCollection(), vInfo);
        for (size_t i = 0; i < vInfo.size(); i++) {
            const int64_t first = (int64_t)slots.slot(vInfo[i].blockID) * GBFK_BLOCK_CELLS;
            const size_t o = i * GBFK_BLOCK_CELLS;
            ok(ctx, gbfk_upload_field(ctx, GBFK_PW, &pw[o], first, GBFK_BLOCK_CELLS), "upload p_w");
            ok(ctx, gbfk_upload_field(ctx, GBFK_PG, &pg[o], first, GBFK_BLOCK_CELLS), "upload p_g");
            ok(ctx, gbfk_upload_field(ctx, GBFK_PHI, &phi[o], first, GBFK_BLOCK_CELLS), "upload phi");
        }
    }

    /* The grid's current leaves (in getBlocksInfo order) and their ghost
     * lists, uploaded if they differ from the device's. */
    std::vector<MRAG::BlockInfo> sync(GridT &g)
    {
        std::vector<MRAG::BlockInfo> vInfo = g.getBlocksInfo();
        bool same = vInfo.size() == ids.size();
        for (size_t i = 0; same && i < vInfo.size(); i++) same = vInfo[i].blockID == ids[i];
        if (!same) upload_topology(g, vInfo);
        return vInfo;
    }

    /* Per leaf of the uploaded topology, the max |detail| of phi. */
    void details(std::vector<double> &det)
    {
        const double t0 = wall_seconds();
        det.resize(ids.size());
        if (!ids.empty()) ok(ctx, gbfk_fwt_details(ctx, &det[0]), "gbfk_fwt_details");
        stats.detail_sweeps++;
        stats.t_details += wall_seconds() - t0;
    }

    int position(int id) const
    {
        std::map<int, int>::const_iterator it = pos_of.find(id);
        if (it == pos_of.end()) throw Error(GBFK_E_INVALID, "ResidentGrid: block is not a leaf on the device");
        return it->second;
    }

    /* phi of every leaf back into the grid's Cells (for a dump). */
    void download_phi(GridT &g)
    {
        std::vector<MRAG::BlockInfo> vInfo = sync(g);
        std::vector<Real> f(vInfo.size() * GBFK_BLOCK_CELLS);
        for (size_t i = 0; i < vInfo.size(); i++)
            ok(ctx, gbfk_download_field(ctx, GBFK_PHI, &f[i * GBFK_BLOCK_CELLS],
                                        (int64_t)slots.slot(vInfo[i].blockID) * GBFK_BLOCK_CELLS, GBFK_BLOCK_CELLS),
               "download phi");
        scatter_phi(f, g.getBlockCollection(), vInfo);
    }

    template <typename IndexT>
    void note(int level, const IndexT *index, double det, double tol, bool refine)
    {
        const double m = fabs(det / tol - 1.0);
        double &mm = refine ? min_margin_refine : min_margin_compress;
        if (m < mm) mm = m;
        if (m <= near_rel) {
            NearDecision d;
            d.adaptation = adaptation;
            d.level = level;
            for (int k = 0; k < 3; k++) d.index[k] = index[k];
            d.detail = det;
            d.tol = tol;
            near.push_back(d);
        }
    }

private:
    int capacity_;

    void upload_topology(GridT &g, const std::vector<MRAG::BlockInfo> &vInfo)
    {
        const double t0 = wall_seconds();
        std::vector<int> sl(vInfo.size());
        for (size_t i = 0; i < vInfo.size(); i++) sl[i] = slots.slot(vInfo[i].blockID);
        flatten_into(topo, vInfo, g.getBoundaryInfo(), &sl);
        const gbfk_ghost_csr csr = topo.csr();
        ok(ctx, gbfk_set_topology(ctx, &topo.blocks[0], (int)topo.blocks.size(), &csr), "gbfk_set_topology");
        ids.resize(vInfo.size());
        pos_of.clear();
        for (size_t i = 0; i < vInfo.size(); i++) {
            ids[i] = vInfo[i].blockID;
            pos_of[ids[i]] = (int)i;
        }
        stats.uploads++;
        stats.t_upload += wall_seconds() - t0;
    }
};


/* The grid's splitter for a resident run (install with
 * grid.setBlockSplitter(new DeviceSplitter<W, BlockCollection<B>, GridT>(&rg));
 * the grid owns it).  BlockSplitter::_split (MRAG/MRAGcore/MRAGBlockSplitter.h:
 * 110-205) creates the children's IDs in one collection.create call, fills
 * them from each parent's lab, erases the parents and reports the IDs; this
 * does the same with the data movement on the device: the children get free
 * slots, one gbfk_split call interpolates all parents (their labs are those
 * of the topology on the device, the grid's topology before the split), then
 * the parents' slots are released. */
template <typename WaveletsType, typename Collection, typename GridT>
class DeviceSplitter : public MRAG::BlockSplitter<WaveletsType, Collection> {
    ResidentGrid<GridT> *rg_;

public:
    explicit DeviceSplitter(ResidentGrid<GridT> *rg) : rg_(rg) {}

    virtual MRAG::RefinementResult split(Collection &collection, MRAG::BoundaryInfo &boundaryInfo,
                                         const MRAG::RefinementPlan &plan, std::vector<MRAG::RefinementReport> &vNewIDs)
    {
        (void)boundaryInfo;
        std::vector<int> vIDs = collection.create(plan.nNewBlocks);
        const int nr = (int)plan.refinements.size();
        std::vector<int> parents(nr), children(8 * (size_t)nr, -1);
        int k = 0;
        for (int r = 0; r < nr; r++) {
            const MRAG::SingleRefinement &ref = *plan.refinements[r];
            parents[r] = rg_->position(ref.block_info_source.blockID);
            if (ref.children.size() != 8) throw Error(GBFK_E_INVALID, "DeviceSplitter: a 3D split has 8 children");
            for (size_t d = 0; d < ref.children.size(); d++, k++) {
                const int *ri = ref.children[d]->relative_index;
                children[ri[0] + 2 * (ri[1] + 2 * ri[2]) + 8 * (size_t)r] = rg_->slots.acquire(vIDs[k]);
            }
        }
        const double t1 = wall_seconds();
        if (nr) ok(rg_->ctx, gbfk_split(rg_->ctx, nr, &parents[0], &children[0]), "gbfk_split");
        const double t2 = wall_seconds();
        for (int r = 0; r < nr; r++) {
            const int id = plan.refinements[r]->block_info_source.blockID;
            rg_->slots.release(id);
            collection.erase(id);
        }
        k = 0;
        for (int r = 0; r < nr; r++) {
            MRAG::RefinementReport rep;
            rep.blockID = plan.refinements[r]->block_info_source.blockID;
            for (size_t d = 0; d < plan.refinements[r]->children.size(); d++) rep.childrenIDs.push_back(vIDs[k++]);
            vNewIDs.push_back(rep);
        }
        rg_->stats.splits += nr;
        rg_->stats.t_split += t2 - t1;
        MRAG::RefinementResult result;
        result.nChildrenBlocks = (int)vIDs.size();
        result.nCollapsedParentBlocks = nr;
        return result;
    }
};

/* The grid's collapser for a resident run (grid.setBlockCollapser(new
 * DeviceCollapser<W, BlockCollection<B>, GridT>(&rg))).
 * BlockCollapser::_collapse (MRAG/MRAGcore/MRAGBlockCollapser.h:100-170)
 * creates one new ID per collapse, fills each parent from its 8 sources by
 * Ha analysis, erases the sources and reports {c, new ID}; the data moves
 * here with one gbfk_collapse call. */
template <typename WaveletsType, typename Collection, typename GridT>
class DeviceCollapser : public MRAG::BlockCollapser<WaveletsType, Collection> {
    ResidentGrid<GridT> *rg_;

public:
    explicit DeviceCollapser(ResidentGrid<GridT> *rg) : rg_(rg) {}

    virtual MRAG::CompressionResult collapse(Collection &collection, MRAG::BoundaryInfo &boundaryInfo,
                                             const MRAG::CompressionPlan &plan,
                                             std::vector<MRAG::BlockCollapseInfo> &vNewIDs)
    {
        (void)boundaryInfo;
        std::vector<int> vIDs = collection.create(plan.nCollapses);
        const int n = plan.nCollapses;
        std::vector<int> parents(n), children(8 * (size_t)n, -1);
        int nCollapsed = 0;
        for (int c = 0; c < n; c++) {
            const MRAG::CompressionPlan::Collapse &col = plan.vCollapseArray[c];
            if (col.nSources != 8) throw Error(GBFK_E_INVALID, "DeviceCollapser: a 3D collapse has 8 sources");
            for (int q = 0; q < col.nSources; q++) {
                const int *a = col.source_index[q].i;
                const int rel = (a[0] & 1) + 2 * ((a[1] & 1) + 2 * (a[2] & 1));
                children[8 * (size_t)c + rel] = rg_->slots.slot(col.source_blockIDs[q]);
            }
            parents[c] = rg_->slots.acquire(vIDs[c]);
            nCollapsed += col.nSources;
        }
        const double t1 = wall_seconds();
        if (n) ok(rg_->ctx, gbfk_collapse(rg_->ctx, n, &children[0], &parents[0]), "gbfk_collapse");
        const double t2 = wall_seconds();
        for (int c = 0; c < n; c++) {
            const MRAG::CompressionPlan::Collapse &col = plan.vCollapseArray[c];
            for (int q = 0; q < col.nSources; q++) {
                rg_->slots.release(col.source_blockIDs[q]);
                collection.erase(col.source_blockIDs[q]);
            }
        }
        for (int c = 0; c < n; c++) {
            MRAG::BlockCollapseInfo bi = {c, vIDs[c]};
            vNewIDs.push_back(bi);
        }
        rg_->stats.collapses += n;
        rg_->stats.t_collapse += t2 - t1;
        MRAG::CompressionResult result = {nCollapsed, (int)vIDs.size()};
        return result;
    }
};

/* Science::AutomaticRefinement (MRAG/MRAGscience/MRAGScienceCore.h:42-106)
 * with the details from the device: blocks below iMaxLevel that are not
 * "nice guys" are refined when their detail is >= the tolerance, else become
 * nice guys; g.refine runs the grid's plan (through DeviceSplitter).  Returns
 * the number of parents split, as the reference does. */
template <typename GridT>
int AutomaticRefinement(GridT &g, ResidentGrid<GridT> &rg, double tol, int iMaxLevel = -1, int iMaxLoops = -1)
{
    std::set<int> niceGuys;
    int loops = 0, nRefined = 0;
    std::vector<double> det;
    while (true) {
        const std::vector<MRAG::BlockInfo> vInfo = rg.sync(g);
        rg.details(det);
        const double t0 = wall_seconds();
        std::set<int> toRefine;
        for (size_t i = 0; i < vInfo.size(); i++) {
            const MRAG::BlockInfo &b = vInfo[i];
            if (iMaxLevel >= 0 && iMaxLevel <= b.level) continue;
            if (niceGuys.count(b.blockID)) continue;
            rg.note(b.level, b.index, det[i], tol, true);
            if (det[i] >= tol) toRefine.insert(b.blockID);
            else niceGuys.insert(b.blockID);
        }
        rg.stats.t_plan += wall_seconds() - t0;
        if (toRefine.empty()) break;
        const double t1 = wall_seconds(), s1 = rg.stats.t_split;
        const MRAG::RefinementResult r = g.refine(toRefine);
        nRefined += r.nCollapsedParentBlocks;
        g.getBoundaryInfo();
        rg.stats.t_plan += (wall_seconds() - t1) - (rg.stats.t_split - s1);
        loops++;
        if (iMaxLoops > 0 && loops >= iMaxLoops) break;
    }
    return nRefined;
}

/* Science::AutomaticCompression (MRAGScienceCore.h:108-177) with the details
 * from the device; g.compress runs the grid's plan (through DeviceCollapser).
 * Returns the number of blocks collapsed. */
template <typename GridT>
int AutomaticCompression(GridT &g, ResidentGrid<GridT> &rg, double tol, int iMaxLoops = -1)
{
    std::set<int> niceGuys;
    int loops = 0, nTotal = 0;
    std::vector<double> det;
    while (true) {
        const std::vector<MRAG::BlockInfo> vInfo = rg.sync(g);
        rg.details(det);
        const double t0 = wall_seconds();
        std::set<int> toCompress;
        for (size_t i = 0; i < vInfo.size(); i++) {
            const MRAG::BlockInfo &b = vInfo[i];
            if (niceGuys.count(b.blockID)) continue;
            rg.note(b.level, b.index, det[i], tol, false);
            if (det[i] < tol) toCompress.insert(b.blockID);
            else niceGuys.insert(b.blockID);
        }
        rg.stats.t_plan += wall_seconds() - t0;
        if (toCompress.empty()) break;
        const double t1 = wall_seconds(), c1 = rg.stats.t_collapse;
        int nCollapsed = 0;
        g.compress(toCompress, nCollapsed);
        g.getBoundaryInfo();
        rg.stats.t_plan += (wall_seconds() - t1) - (rg.stats.t_collapse - c1);
        if (nCollapsed == 0) break;
        nTotal += nCollapsed;
        loops++;
        if (iMaxLoops > 0 && loops >= iMaxLoops) break;
    }
    return nTotal;
}

}  // namespace gbfk_mrag
