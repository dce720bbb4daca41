// C ABI of the gbfk library (include/gbfk.h): context, topology, data
// movement and the hot-path entry points.  Host code only; kernels live in
// gbfk_kernels.cu.
#include "gbfk.h"
#include "gbfk_kernels.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

namespace gbfk {
cudaError_t upload_ghost_table();
void init_ghost_table_host(short *table);
}  // namespace gbfk

using namespace gbfk;

struct gbfk_ctx {
    int precision = GBFK_F64;
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int max_blocks = 0;
    size_t rsize = 8;  // sizeof(Real)

    // block pool (Real): phi is double-buffered across steps
    void *phi[2] = {nullptr, nullptr};
    int cur = 0;
    void *pw = nullptr, *pg = nullptr;

    // topology
    int nblocks = 0;
    bool have_topology = false;
    bool uniform = false;
    int bpd = 0;
    std::vector<int> h_slot;
    std::vector<double> h_h;
    int *d_slot = nullptr;
    int *d_nbr = nullptr;
    void *d_h = nullptr;
    // ghost CSR (rows = nblocks * 488)
    bool have_csr = false;
    int64_t nrows = 0;
    int64_t *d_row_ptr = nullptr;
    int *d_src = nullptr;
    void *d_w = nullptr;
    int *d_step_rows = nullptr;
    int64_t n_step_rows = 0;
    int *d_all_rows = nullptr;
    void *d_gpw = nullptr, *d_gpg = nullptr, *d_gphi = nullptr;
    bool static_ghosts_dirty = true;

    // static per (topology, p_w, p_g): cell classes; per (.., Dw, Dg): face coefficients
    void *d_origin = nullptr;         // nblocks * 3 Real: BlockInfo::origin
    bool have_origin = false;
    // capacity in bytes of each topology buffer (keyed by the member's
    // address): the buffers are kept across topology changes and grown only
    // when a topology needs more room
    std::unordered_map<void *, size_t> topo_cap;

    // observations for the likelihood (n^3 grid)
    int obs_n = 0;
    unsigned char *d_t1c = nullptr, *d_flair = nullptr;
    double *d_pet = nullptr;
    int *d_roi = nullptr;
    int nroi = 0;
    double *d_model = nullptr;        // dump grid
    size_t model_bytes = 0;
    double *d_partial = nullptr;      // likelihood partial sums
    double *d_lik = nullptr;          // 4 results
    int *d_roi_count = nullptr;       // n^3: how often the ROI lists each voxel (the adjoint's loss weights)
    size_t roi_count_bytes = 0;

    unsigned short *d_meta = nullptr; // max_blocks * 512 meta words, indexed like the pool
    unsigned char *d_btype = nullptr; // nblocks block types
    bool identity_slots = false;
    void *d_H = nullptr;              // nblocks * 1728 Real
    double *d_ih2 = nullptr;          // nblocks: 1/(h*h) in double
    bool faces_valid = false;
    double faces_Dw = 0, faces_Dg = 0;

    // step kernel: preference (GBFK_STEP_*), the one the last step ran, and
    // the pipelined step's tensor maps of phi[0] / phi[1]
    int step_pref = GBFK_STEP_AUTO;
    int step_used = 0;
    bool tma_maps_ready = false;
    CUtensorMap tma_maps[2][3];
    // the pipelined step's work lists (heavy blocks, then empty blocks), from d_btype
    int *d_lists = nullptr;
    int n_heavy = 0, n_empty = 0;
    bool lists_valid = false;
    std::vector<int> h_lists;  // host copy of d_lists
    // runs of steps in one launch: the CTA count, per CTA the CTAs that own
    // face neighbours of its blocks (d_run_nbr: offsets, then the lists) and
    // the step flags
    int run_ctas = 0;
    bool run_layout_valid = false;
    int *d_run_nbr = nullptr;
    unsigned *d_run_flags = nullptr;
    // phi[cur] is the output of a step: every value +0 <= phi <= 1 or NaN
    // (set only by rd_step; every other writer of phi clears it)
    bool phi_clamped = false;

    // scratch
    unsigned *d_nan = nullptr;        // [0]: NaN seen in a step, [1]: a pipeline stage wait timed out
    void *d_stage = nullptr;
    size_t stage_bytes = 0;
    // gbfk_forward_adjoint's device buffers, kept from one call to the next
    // (freed by gbfk_destroy, or replaced when a call needs other sizes or
    // more checkpoint buffers)
    std::vector<void *> adj_mem;
    size_t adj_fbytes = 0;
    int adj_nblocks = 0, adj_nsnap = 0;
    // the adjoint's state buffers whose empty blocks hold +0 (forward steps
    // into them may skip those blocks), valid for the step lists of
    // generation adj_clean_gen
    std::unordered_set<const void *> adj_clean;
    int64_t lists_gen = 0, adj_clean_gen = -1;
    // the forward steps of gbfk_forward_adjoint run on adj_fstream, the
    // adjoint steps on `stream`; per state buffer one event for its last
    // forward write and one for its last adjoint read, and a fork/join event
    cudaStream_t adj_fstream = nullptr;
    std::unordered_map<const void *, cudaEvent_t> adj_ev_write, adj_ev_read;
    cudaEvent_t adj_ev_join = nullptr;
    // gbfk_rd_step_host: an input and an output copy stream, two sets of
    // staging buffers and their events (set k & 1 serves call k)
    cudaStream_t io_in_stream = nullptr, io_out_stream = nullptr;
    void *io_in[2] = {nullptr, nullptr}, *io_out[2] = {nullptr, nullptr};
    size_t io_bytes = 0;
    cudaEvent_t io_ev[4][2] = {};  // in ready, in free, out ready, out free
    bool io_ready = false;
    int64_t io_calls = 0;
    double *d_fwt = nullptr;
    int *d_ints = nullptr;
    size_t ints_cap = 0;

    int64_t launches = 0;
    std::string err;
};

namespace {

int fail(gbfk_ctx *c, int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    return code;
}

#define CK(call)                                                                                      \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess)                                                                        \
            return fail(ctx, e_ == cudaErrorMemoryAllocation ? GBFK_E_OOM : GBFK_E_CUDA, "%s: %s (%s:%d)", \
                        #call, cudaGetErrorString(e_), __FILE__, __LINE__);                           \
    } while (0)

std::mutex g_table_mutex;
std::vector<int> g_table_ready;  // per device

int ensure_table(gbfk_ctx *ctx)
{
    std::lock_guard<std::mutex> lk(g_table_mutex);
    if ((int)g_table_ready.size() <= ctx->device) g_table_ready.resize(ctx->device + 1, 0);
    if (!g_table_ready[ctx->device]) {
        CK(upload_ghost_table());
        g_table_ready[ctx->device] = 1;
    }
    return GBFK_OK;
}

// A topology buffer of at least `bytes`: the one already held if it is large
// enough, else a new one (the old contents are not kept).
template <typename T>
int topo_alloc(gbfk_ctx *c, T **p, size_t bytes)
{
    void **q = (void **)p;
    bytes = std::max<size_t>(bytes, 1);
    auto it = c->topo_cap.find((void *)q);
    if (*q && it != c->topo_cap.end() && it->second >= bytes) return GBFK_OK;
    if (*q) cudaFree(*q);
    *q = nullptr;
    c->topo_cap.erase((void *)q);
    const cudaError_t e = cudaMalloc(q, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(c, GBFK_E_OOM, "topology buffer of %zu bytes: %s", bytes, cudaGetErrorString(e));
    }
    c->topo_cap[(void *)q] = bytes;
    return GBFK_OK;
}

// Forget the current topology; its buffers stay allocated for the next one.
void free_topology(gbfk_ctx *c)
{
    c->have_topology = c->have_csr = c->uniform = c->have_origin = false;
    c->nblocks = 0;
    c->nrows = c->n_step_rows = 0;
    c->h_slot.clear();
    c->h_h.clear();
    c->static_ghosts_dirty = true;
    c->faces_valid = false;
    c->lists_valid = false;
    c->run_layout_valid = false;
    c->phi_clamped = false;
}

// Free the topology buffers (context destruction).
void release_topology(gbfk_ctx *c)
{
    free_topology(c);
    void **ptrs[] = {(void **)&c->d_slot, (void **)&c->d_nbr, &c->d_h, (void **)&c->d_row_ptr, (void **)&c->d_src,
                     &c->d_w, (void **)&c->d_step_rows, (void **)&c->d_all_rows, &c->d_gpw, &c->d_gpg,
                     &c->d_gphi, (void **)&c->d_fwt, &c->d_H, (void **)&c->d_ih2, (void **)&c->d_btype, &c->d_origin,
                     (void **)&c->d_lists, (void **)&c->d_run_nbr, (void **)&c->d_run_flags};
    for (void **p : ptrs) {
        if (*p) cudaFree(*p);
        *p = nullptr;
    }
    c->topo_cap.clear();
}

// Something the face coefficients or classes depend on changed.
void invalidate_static(gbfk_ctx *c)
{
    c->static_ghosts_dirty = true;
    c->faces_valid = false;
}

// Per-block BlockInfo::origin = index * 2^-level in Real (MRAGrid.inl:208-212).
int upload_origin(gbfk_ctx *ctx, const std::vector<int> &level, const std::vector<int> &index)
{
    const int nb = ctx->nblocks;
    std::vector<double> o(3 * (size_t)nb);
    for (int i = 0; i < nb; i++)
        for (int d = 0; d < 3; d++) o[3 * i + d] = index[3 * i + d] * ldexp(1.0, -level[i]);
    {
        const int rc = topo_alloc(ctx, &ctx->d_origin, 3 * (size_t)nb * ctx->rsize);
        if (rc) return rc;
    }
    if (ctx->precision == GBFK_F64) {
        CK(cudaMemcpy(ctx->d_origin, o.data(), o.size() * sizeof(double), cudaMemcpyHostToDevice));
    } else {
        std::vector<float> f(o.begin(), o.end());
        CK(cudaMemcpy(ctx->d_origin, f.data(), f.size() * sizeof(float), cudaMemcpyHostToDevice));
    }
    ctx->have_origin = true;
    return GBFK_OK;
}

// Per-block 1/(h*h) in double, as the operator forms it (ReactionDiffusionOperator.h:49-50).
int upload_ih2(gbfk_ctx *ctx)
{
    std::vector<double> v(ctx->nblocks);
    for (int i = 0; i < ctx->nblocks; i++) {
        const double h = ctx->precision == GBFK_F64 ? ctx->h_h[i] : (double)(float)ctx->h_h[i];
        v[i] = 1. / (h * h);
    }
    {
        const int rc = topo_alloc(ctx, &ctx->d_ih2, ctx->nblocks * sizeof(double));
        if (rc) return rc;
    }
    CK(cudaMemcpy(ctx->d_ih2, v.data(), ctx->nblocks * sizeof(double), cudaMemcpyHostToDevice));
    return GBFK_OK;
}

template <typename Real>
PoolView<Real> view(gbfk_ctx *c)
{
    PoolView<Real> v;
    v.slot = c->d_slot;
    v.nbr = c->d_nbr;
    v.hblk = (const Real *)c->d_h;
    v.gpw = (const Real *)c->d_gpw;
    v.gpg = (const Real *)c->d_gpg;
    v.gphi = (const Real *)c->d_gphi;
    v.pw = (const Real *)c->pw;
    v.pg = (const Real *)c->pg;
    v.btype = c->d_btype;
    v.nblocks = c->nblocks;
    v.identity_slots = c->identity_slots ? 1 : 0;
    v.log2_bpd = -1;
    if (c->uniform && !c->have_csr && (c->bpd & (c->bpd - 1)) == 0) {
        int L = 0;
        while ((1 << L) < c->bpd) L++;
        v.log2_bpd = L;
    }
    return v;
}

int ints_scratch(gbfk_ctx *ctx, size_t n)
{
    if (ctx->ints_cap >= n) return GBFK_OK;
    if (ctx->d_ints) cudaFree(ctx->d_ints);
    ctx->d_ints = nullptr;
    ctx->ints_cap = 0;
    CK(cudaMalloc(&ctx->d_ints, n * sizeof(int)));
    ctx->ints_cap = n;
    return GBFK_OK;
}

// The pipelined step's error word (d_nan[1]: bit 0 a wait timed out, bit 1 a
// work list overflowed, bits 3-8 the wait that timed out: launch_rd_run_tma);
// reading it synchronises the stream.  An error is reported once and the
// word cleared.
int check_stage_timeout(gbfk_ctx *ctx)
{
    unsigned flag = 0;
    CK(cudaMemcpyAsync(&flag, ctx->d_nan + 1, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (flag) {
        CK(cudaMemsetAsync(ctx->d_nan + 1, 0, sizeof(unsigned), ctx->stream));
        if (flag & (1u | 256u))
            return fail(ctx, GBFK_E_TIMEOUT, "rd_step: a wait of the pipelined step timed out (1 s; error word 0x%x)",
                        flag);
        return fail(ctx, GBFK_E_CUDA, "rd_step: a CTA's work list of the pipelined step overflowed");
    }
    return GBFK_OK;
}

// Lab positions of face f (0..5) in face_cell order, with the source cell in
// the same-level neighbour.
void face_positions(int f, int p, int &lx, int &ly, int &lz, int &src_cell)
{
    const int a = p & 7, b = p >> 3;
    const int d = f >> 1, plus = f & 1;
    const int c_lab = plus ? kBS : -1;
    const int c_src = plus ? 0 : kBS - 1;
    if (d == 0) { lx = c_lab; ly = a; lz = b; src_cell = c_src + kBS * (a + kBS * b); }
    else if (d == 1) { lx = a; ly = c_lab; lz = b; src_cell = a + kBS * (c_src + kBS * b); }
    else { lx = a; ly = b; lz = c_lab; src_cell = a + kBS * (b + kBS * c_src); }
}

inline int lab_idx(int x, int y, int z) { return (x + 1) + kLab * ((y + 1) + kLab * (z + 1)); }

template <typename Real>
int set_csr(gbfk_ctx *ctx, const int64_t *row_ptr, const std::vector<int> &src, const double *w0, const double *w1,
            const double *w2, bool detect_direct)
{
    const int nb = ctx->nblocks;
    const int64_t nrows = (int64_t)nb * kLabGhosts;
    const int64_t nnz = row_ptr[nrows];
    std::vector<Real> w(nnz);
    for (int64_t k = 0; k < nnz; k++) w[k] = ((Real)w0[k] * (Real)w1[k]) * (Real)w2[k];

    short table[kLab3];
    init_ghost_table_host(table);

    // same-level faces: every row one entry of weight 1 from one neighbour
    std::vector<int> nbr((size_t)nb * 6, -1);
    std::vector<int> step_rows;
    for (int b = 0; b < nb; b++) {
        for (int f = 0; f < 6; f++) {
            int nb_slot = -2;
            bool direct = detect_direct;
            for (int p = 0; p < kFaceCells && direct; p++) {
                int lx, ly, lz, sc;
                face_positions(f, p, lx, ly, lz, sc);
                const int64_t r = (int64_t)b * kLabGhosts + table[lab_idx(lx, ly, lz)];
                if (row_ptr[r + 1] - row_ptr[r] != 1) { direct = false; break; }
                const int64_t k = row_ptr[r];
                if (!(w[k] == (Real)1)) { direct = false; break; }
                const int s = src[k] / kBS3, cell = src[k] % kBS3;
                if (cell != sc) { direct = false; break; }
                if (nb_slot == -2) nb_slot = s;
                else if (nb_slot != s) { direct = false; break; }
            }
            if (direct) {
                nbr[(size_t)b * 6 + f] = nb_slot;
            } else {
                for (int p = 0; p < kFaceCells; p++) {
                    int lx, ly, lz, sc;
                    face_positions(f, p, lx, ly, lz, sc);
                    step_rows.push_back(b * kLabGhosts + table[lab_idx(lx, ly, lz)]);
                }
            }
        }
    }
    std::vector<int> all_rows(nrows);
    for (int64_t r = 0; r < nrows; r++) all_rows[r] = (int)r;

    int rc = GBFK_OK;
    if (!rc) rc = topo_alloc(ctx, &ctx->d_row_ptr, (nrows + 1) * sizeof(int64_t));
    if (!rc) rc = topo_alloc(ctx, &ctx->d_src, std::max<int64_t>(nnz, 1) * sizeof(int));
    if (!rc) rc = topo_alloc(ctx, &ctx->d_w, std::max<int64_t>(nnz, 1) * sizeof(Real));
    if (!rc) rc = topo_alloc(ctx, &ctx->d_nbr, (size_t)nb * 6 * sizeof(int));
    if (!rc) rc = topo_alloc(ctx, &ctx->d_all_rows, nrows * sizeof(int));
    if (!rc) rc = topo_alloc(ctx, &ctx->d_step_rows, std::max<size_t>(step_rows.size(), 1) * sizeof(int));
    if (!rc) rc = topo_alloc(ctx, &ctx->d_gpw, nrows * sizeof(Real));
    if (!rc) rc = topo_alloc(ctx, &ctx->d_gpg, nrows * sizeof(Real));
    if (!rc) rc = topo_alloc(ctx, &ctx->d_gphi, nrows * sizeof(Real));
    if (rc) return rc;
    CK(cudaMemcpy(ctx->d_row_ptr, row_ptr, (nrows + 1) * sizeof(int64_t), cudaMemcpyHostToDevice));
    if (nnz) {
        CK(cudaMemcpy(ctx->d_src, src.data(), nnz * sizeof(int), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(ctx->d_w, w.data(), nnz * sizeof(Real), cudaMemcpyHostToDevice));
    }
    CK(cudaMemcpy(ctx->d_nbr, nbr.data(), (size_t)nb * 6 * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->d_all_rows, all_rows.data(), nrows * sizeof(int), cudaMemcpyHostToDevice));
    if (!step_rows.empty())
        CK(cudaMemcpy(ctx->d_step_rows, step_rows.data(), step_rows.size() * sizeof(int), cudaMemcpyHostToDevice));
    ctx->n_step_rows = (int64_t)step_rows.size();
    ctx->nrows = nrows;
    ctx->have_csr = true;
    invalidate_static(ctx);
    return GBFK_OK;
}

// Same-level periodic ghost lists of a uniform grid, as the reference's
// BBInfoCreator builds them for equal-level neighbours (one entry, weights
// 1*1*1), so that the ghost-reading kernels (details, split) work on it.
int build_uniform_csr(gbfk_ctx *ctx)
{
    const int bpd = ctx->bpd, nb = ctx->nblocks;
    short table[kLab3];
    init_ghost_table_host(table);
    const int64_t nrows = (int64_t)nb * kLabGhosts;
    std::vector<int64_t> row_ptr(nrows + 1);
    std::vector<int> src(nrows);
    std::vector<double> ones(nrows, 1.0);
    for (int64_t r = 0; r <= nrows; r++) row_ptr[r] = r;
    for (int bz = 0; bz < bpd; bz++)
        for (int by = 0; by < bpd; by++)
            for (int bx = 0; bx < bpd; bx++) {
                const int b = bx + bpd * (by + bpd * bz);
                for (int z = -1; z < 9; z++)
                    for (int y = -1; y < 9; y++)
                        for (int x = -1; x < 9; x++) {
                            const int g = table[lab_idx(x, y, z)];
                            if (g < 0) continue;
                            const int gx = bx * 8 + x, gy = by * 8 + y, gz = bz * 8 + z;
                            const int n = bpd * 8;
                            const int wx = (gx + n) % n, wy = (gy + n) % n, wz = (gz + n) % n;
                            const int sb = (wx >> 3) + bpd * ((wy >> 3) + bpd * (wz >> 3));
                            src[(int64_t)b * kLabGhosts + g] = sb * kBS3 + (wx & 7) + 8 * ((wy & 7) + 8 * (wz & 7));
                        }
            }
    return ctx->precision == GBFK_F64
               ? set_csr<double>(ctx, row_ptr.data(), src, ones.data(), ones.data(), ones.data(), true)
               : set_csr<float>(ctx, row_ptr.data(), src, ones.data(), ones.data(), ones.data(), true);
}

template <typename Real>
int refresh_static_ghosts(gbfk_ctx *ctx)
{
    if (!ctx->have_csr || !ctx->static_ghosts_dirty) return GBFK_OK;
    CK(launch_fill_ghosts<Real>(ctx->d_all_rows, ctx->nrows, ctx->d_row_ptr, ctx->d_src, (const Real *)ctx->d_w,
                                (const Real *)ctx->pw, (Real *)ctx->d_gpw, ctx->stream));
    CK(launch_fill_ghosts<Real>(ctx->d_all_rows, ctx->nrows, ctx->d_row_ptr, ctx->d_src, (const Real *)ctx->d_w,
                                (const Real *)ctx->pg, (Real *)ctx->d_gpg, ctx->stream));
    ctx->launches += 2;
    ctx->static_ghosts_dirty = false;
    return GBFK_OK;
}

// Ghosts of p_w/p_g, cell classes and the face coefficients for (Dw, Dg):
// everything of a step that does not depend on phi.
template <typename Real>
int prepare_static(gbfk_ctx *ctx, double Dw, double Dg)
{
    int rc = refresh_static_ghosts<Real>(ctx);
    if (rc) return rc;
    const double kDw = (double)(Real)Dw, kDg = (double)(Real)Dg;
    if (!ctx->faces_valid || ctx->faces_Dw != kDw || ctx->faces_Dg != kDg) {
        int rc = topo_alloc(ctx, &ctx->d_H, (size_t)ctx->nblocks * kFacesPerBlock * sizeof(Real));
        if (!rc) rc = topo_alloc(ctx, &ctx->d_btype, (size_t)ctx->nblocks);
        if (rc) return rc;
        CK(launch_faces<Real>(view<Real>(ctx), (Real)Dw, (Real)Dg, (Real *)ctx->d_H, ctx->d_meta, ctx->d_btype,
                              ctx->stream));
        ctx->launches++;
        ctx->faces_valid = true;
        ctx->lists_valid = false;  // block types recomputed
        ctx->faces_Dw = kDw;
        ctx->faces_Dg = kDg;
    }
    return GBFK_OK;
}

// Work lists of the pipelined step from the block types: heavy blocks
// (entry block * 4 + type; mixed blocks first, then tissue blocks), then
// empty blocks (entry: block).  Rebuilt whenever the block types change.
int build_step_lists(gbfk_ctx *ctx)
{
    if (ctx->lists_valid) return GBFK_OK;
    const int nb = ctx->nblocks;
    std::vector<unsigned char> bt(nb);
    CK(cudaMemcpyAsync(bt.data(), ctx->d_btype, nb, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    std::vector<int> lists;
    lists.reserve(nb);
    for (int b = 0; b < nb; b++)
        if (bt[b] == kBlockMixed) lists.push_back(b * 4 + kBlockMixed);
    for (int b = 0; b < nb; b++)
        if (bt[b] == kBlockTissue) lists.push_back(b * 4 + kBlockTissue);
    const int nh = (int)lists.size();
    for (int b = 0; b < nb; b++)
        if (bt[b] == kBlockEmpty) lists.push_back(b);
    if ((int)lists.size() != nb) return fail(ctx, GBFK_E_CUDA, "rd_step: unknown block type");
    {
        const int rc = topo_alloc(ctx, &ctx->d_lists, (size_t)nb * sizeof(int));
        if (rc) return rc;
    }
    CK(cudaMemcpyAsync(ctx->d_lists, lists.data(), (size_t)nb * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->n_heavy = nh;
    ctx->n_empty = nb - nh;
    ctx->lists_valid = true;
    ctx->lists_gen++;
    ctx->h_lists.swap(lists);
    ctx->run_layout_valid = false;
    return GBFK_OK;
}

// The CTA layout of runs of steps over the current step lists.
template <typename Real>
int build_run_layout(gbfk_ctx *ctx, const PoolView<Real> &v)
{
    if (ctx->run_layout_valid) return GBFK_OK;
    std::vector<int> off, nbr;
    int G = 0;
    CK(rd_run_layout<Real>(v, ctx->h_lists.data(), ctx->n_heavy, ctx->h_lists.data() + ctx->n_heavy, ctx->n_empty, G,
                           off, nbr));
    off.insert(off.end(), nbr.begin(), nbr.end());
    int rc = topo_alloc(ctx, &ctx->d_run_nbr, off.size() * sizeof(int));
    if (!rc) rc = topo_alloc(ctx, &ctx->d_run_flags, (size_t)G * kRunFlagStride * sizeof(unsigned));
    if (rc) return rc;
    CK(cudaMemcpyAsync(ctx->d_run_nbr, off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->run_ctas = G;
    ctx->run_layout_valid = true;
    return GBFK_OK;
}

template <typename Real>
int rd_step_impl(gbfk_ctx *ctx, double Dw, double Dg, double rho, double dt, int nsteps, int check_nan)
{
    int rc = prepare_static<Real>(ctx, Dw, Dg);
    if (rc) return rc;
    PoolView<Real> v = view<Real>(ctx);
    const bool eligible = tma_step_eligible<Real>(v);
    if ((ctx->step_pref == GBFK_STEP_PIPELINED || ctx->step_pref == GBFK_STEP_RUN) && !eligible)
        return fail(ctx, GBFK_E_STATE, "rd_step: the pipelined step needs a uniform power-of-two grid (gbfk_set_uniform)");
    const bool pipelined = eligible && ctx->step_pref != GBFK_STEP_BLOCK;
    // runs of steps in one launch: on request only (on B200 they are within
    // a few percent of one launch per step, which programmatic dependent
    // launch already overlaps)
    const bool runs = pipelined && ctx->step_pref == GBFK_STEP_RUN;
    double ih2 = 0;
    if (pipelined) {
        if (!ctx->tma_maps_ready) {
            for (int b = 0; b < 2; b++)
                CK(make_pool_tensor_maps(ctx->phi[b], ctx->max_blocks, (int)sizeof(Real), ctx->tma_maps[b]));
            ctx->tma_maps_ready = true;
        }
        rc = build_step_lists(ctx);
        if (!rc && runs) rc = build_run_layout<Real>(ctx, v);
        if (rc) return rc;
        // uniform grid: one h for every block, as upload_ih2 forms it
        const double h = sizeof(Real) == 8 ? ctx->h_h[0] : (double)(float)ctx->h_h[0];
        ih2 = 1. / (h * h);
    }
    if (check_nan) CK(cudaMemsetAsync(ctx->d_nan, 0, sizeof(unsigned), ctx->stream));
    const BlockLists lists = {ctx->d_lists, ctx->n_heavy, ctx->d_lists + ctx->n_heavy, ctx->n_empty};
    bool ran_run = false;
    for (int s = 0; s < nsteps;) {
        const Real *in = (const Real *)ctx->phi[ctx->cur];
        Real *out = (Real *)ctx->phi[ctx->cur ^ 1];
        const bool clamped = ctx->phi_clamped || s > 0;
        const int left = nsteps - s;
        if (runs && clamped && left >= 2) {
            // phi[cur] -> phi[cur ^ 1] -> phi[cur] ..., k steps in one launch
            const int k = left < kMaxRunSteps ? left : kMaxRunSteps;
            Real *last = (Real *)ctx->phi[ctx->cur ^ (k & 1)];
            CK(launch_rd_run_tma<Real>(v, lists, ctx->run_ctas, ctx->d_run_nbr, ctx->d_run_nbr + ctx->run_ctas + 1,
                                       (const Real *)ctx->d_H, ctx->d_meta, ih2, in, out, (Real *)ctx->phi[ctx->cur],
                                       last, k, (Real)rho, dt, ctx->d_nan, ctx->d_nan + 1, ctx->d_run_flags,
                                       ctx->tma_maps[ctx->cur], ctx->tma_maps[ctx->cur ^ 1], ctx->tma_maps[ctx->cur],
                                       ctx->stream));
            ctx->launches++;
            ctx->cur ^= (k & 1);
            s += k;
            ran_run = true;
            continue;
        }
        if (pipelined) {
            CK(launch_rd_step_tma<Real>(v, lists, (const Real *)ctx->d_H, ctx->d_meta, ih2, in, clamped, out,
                                        (Real)rho, dt, ctx->d_nan, ctx->d_nan + 1, ctx->tma_maps[ctx->cur], false,
                                        ctx->stream));
            ctx->launches++;
            ctx->cur ^= 1;
            s++;
            continue;
        }
        if (ctx->n_step_rows > 0) {
            CK(launch_fill_ghosts<Real>(ctx->d_step_rows, ctx->n_step_rows, ctx->d_row_ptr, ctx->d_src,
                                        (const Real *)ctx->d_w, in, (Real *)ctx->d_gphi, ctx->stream));
            ctx->launches++;
        }
        CK(launch_rd_step<Real>(v, (const Real *)ctx->d_H, ctx->d_meta, ctx->d_ih2, in, out, nullptr, (Real)rho, dt,
                                ctx->d_nan, ctx->stream));
        ctx->launches++;
        ctx->cur ^= 1;
        s++;
    }
    if (nsteps > 0) {
        ctx->step_used = ran_run ? GBFK_STEP_RUN : pipelined ? GBFK_STEP_PIPELINED : GBFK_STEP_BLOCK;
        ctx->phi_clamped = true;
    }
    if (check_nan) {
        unsigned flag = 0;
        CK(cudaMemcpyAsync(&flag, ctx->d_nan, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        int rc2 = check_stage_timeout(ctx);
        if (rc2) return rc2;
        if (flag) return fail(ctx, GBFK_E_NAN, "phi became NaN during the step");
    }
    return GBFK_OK;
}

template <typename Real>
int rd_rhs_impl(gbfk_ctx *ctx, double Dw, double Dg, double rho, void *host)
{
    int rc = prepare_static<Real>(ctx, Dw, Dg);
    if (rc) return rc;
    const size_t bytes = (size_t)ctx->nblocks * kBS3 * sizeof(Real);
    Real *d_out = nullptr;
    CK(cudaMalloc(&d_out, bytes));
    PoolView<Real> v = view<Real>(ctx);
    const Real *in = (const Real *)ctx->phi[ctx->cur];
    cudaError_t e = cudaSuccess;
    if (ctx->n_step_rows > 0) {
        e = launch_fill_ghosts<Real>(ctx->d_step_rows, ctx->n_step_rows, ctx->d_row_ptr, ctx->d_src,
                                     (const Real *)ctx->d_w, in, (Real *)ctx->d_gphi, ctx->stream);
        ctx->launches++;
    }
    if (e == cudaSuccess) {
        e = launch_rd_step<Real>(v, (const Real *)ctx->d_H, ctx->d_meta, ctx->d_ih2, in, nullptr, d_out, (Real)rho,
                                 0.0, ctx->d_nan, ctx->stream);
        ctx->launches++;
    }
    // dphidt leaves in topology order: block i's 512 cells at i*512
    if (e == cudaSuccess) {
        for (int i = 0; i < ctx->nblocks && e == cudaSuccess; i++)
            e = cudaMemcpyAsync((char *)host + (size_t)i * kBS3 * sizeof(Real),
                                (const char *)d_out + (size_t)ctx->h_slot[i] * kBS3 * sizeof(Real),
                                kBS3 * sizeof(Real), cudaMemcpyDeviceToHost, ctx->stream);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(d_out);
    CK(e);
    return GBFK_OK;
}

template <typename Real>
int fwt_impl(gbfk_ctx *ctx, double *out)
{
    if (!ctx->have_csr && ctx->uniform) {
        int rc = build_uniform_csr(ctx);
        if (rc) return rc;
    }
    int rc = refresh_static_ghosts<Real>(ctx);
    if (rc) return rc;
    const Real *phi = (const Real *)ctx->phi[ctx->cur];
    CK(launch_fill_ghosts<Real>(ctx->d_all_rows, ctx->nrows, ctx->d_row_ptr, ctx->d_src, (const Real *)ctx->d_w,
                                phi, (Real *)ctx->d_gphi, ctx->stream));
    {
        const int rc = topo_alloc(ctx, &ctx->d_fwt, (size_t)ctx->nblocks * sizeof(double));
        if (rc) return rc;
    }
    CK(launch_fwt_details<Real>(view<Real>(ctx), phi, ctx->d_fwt, ctx->stream));
    ctx->launches += 2;
    CK(cudaMemcpyAsync(out, ctx->d_fwt, (size_t)ctx->nblocks * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return GBFK_OK;
}

template <typename Real>
int split_impl(gbfk_ctx *ctx, int nsplit, const int *parents, const int *children)
{
    ctx->phi_clamped = false;  // the interpolation may leave [0, 1]
    if (!ctx->have_csr && ctx->uniform) {
        int rc = build_uniform_csr(ctx);
        if (rc) return rc;
    }
    int rc = refresh_static_ghosts<Real>(ctx);
    if (rc) return rc;
    for (int i = 0; i < nsplit; i++) {
        if (parents[i] < 0 || parents[i] >= ctx->nblocks)
            return fail(ctx, GBFK_E_INVALID, "split: parent %d is not a block of the topology", parents[i]);
        for (int c = 0; c < 8; c++)
            if (children[8 * i + c] < 0 || children[8 * i + c] >= ctx->max_blocks)
                return fail(ctx, GBFK_E_INVALID, "split: child slot %d out of range", children[8 * i + c]);
    }
    const Real *phi = (const Real *)ctx->phi[ctx->cur];
    CK(launch_fill_ghosts<Real>(ctx->d_all_rows, ctx->nrows, ctx->d_row_ptr, ctx->d_src, (const Real *)ctx->d_w,
                                phi, (Real *)ctx->d_gphi, ctx->stream));
    rc = ints_scratch(ctx, (size_t)nsplit * 9);
    if (rc) return rc;
    CK(cudaMemcpyAsync(ctx->d_ints, parents, nsplit * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->d_ints + nsplit, children, (size_t)nsplit * 8 * sizeof(int), cudaMemcpyHostToDevice,
                       ctx->stream));
    CK(launch_split<Real>(view<Real>(ctx), nsplit, ctx->d_ints, ctx->d_ints + nsplit, (Real *)ctx->phi[ctx->cur],
                          (Real *)ctx->pw, (Real *)ctx->pg, ctx->stream));
    ctx->launches += 2;
    invalidate_static(ctx);
    CK(cudaStreamSynchronize(ctx->stream));
    return GBFK_OK;
}

template <typename Real>
int collapse_impl(gbfk_ctx *ctx, int n, const int *children, const int *parents)
{
    ctx->phi_clamped = false;
    for (int i = 0; i < n; i++) {
        if (parents[i] < 0 || parents[i] >= ctx->max_blocks)
            return fail(ctx, GBFK_E_INVALID, "collapse: parent slot %d out of range", parents[i]);
        for (int c = 0; c < 8; c++)
            if (children[8 * i + c] < 0 || children[8 * i + c] >= ctx->max_blocks)
                return fail(ctx, GBFK_E_INVALID, "collapse: child slot %d out of range", children[8 * i + c]);
    }
    int rc = ints_scratch(ctx, (size_t)n * 9);
    if (rc) return rc;
    CK(cudaMemcpyAsync(ctx->d_ints, children, (size_t)n * 8 * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->d_ints + (size_t)n * 8, parents, n * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    CK(launch_collapse<Real>(n, ctx->d_ints, ctx->d_ints + (size_t)n * 8, (Real *)ctx->phi[ctx->cur],
                             (Real *)ctx->pw, (Real *)ctx->pg, ctx->stream));
    ctx->launches++;
    invalidate_static(ctx);
    CK(cudaStreamSynchronize(ctx->stream));
    return GBFK_OK;
}

void *field_ptr(gbfk_ctx *c, int field)
{
    switch (field) {
    case GBFK_PHI: return c->phi[c->cur];
    case GBFK_PW: return c->pw;
    case GBFK_PG: return c->pg;
    default: return nullptr;
    }
}

}  // namespace

// ---------------------------------------------------------------------------
extern "C" {

int gbfk_create(const gbfk_config *cfg, gbfk_ctx **out)
{
    if (!cfg || !out) return GBFK_E_INVALID;
    *out = nullptr;
    if (cfg->precision != GBFK_F64 && cfg->precision != GBFK_F32) return GBFK_E_INVALID;
    if (cfg->max_blocks <= 0 || (int64_t)cfg->max_blocks * kBS3 > INT32_MAX) return GBFK_E_INVALID;
    gbfk_ctx *ctx = new gbfk_ctx();
    ctx->precision = cfg->precision;
    ctx->rsize = cfg->precision == GBFK_F64 ? sizeof(double) : sizeof(float);
    ctx->device = cfg->device;
    ctx->max_blocks = cfg->max_blocks;
    auto bail = [&](int rc) {
        gbfk_destroy(ctx);
        return rc;
    };
    if (cudaSetDevice(cfg->device) != cudaSuccess) return bail(GBFK_E_CUDA);
    if (cfg->stream) {
        ctx->stream = (cudaStream_t)cfg->stream;
    } else {
        if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(GBFK_E_CUDA);
        ctx->own_stream = true;
    }
    const size_t bytes = (size_t)cfg->max_blocks * kBS3 * ctx->rsize;
    if (cudaMalloc(&ctx->phi[0], bytes) != cudaSuccess || cudaMalloc(&ctx->phi[1], bytes) != cudaSuccess ||
        cudaMalloc(&ctx->pw, bytes) != cudaSuccess || cudaMalloc(&ctx->pg, bytes) != cudaSuccess ||
        cudaMalloc(&ctx->d_nan, 2 * sizeof(unsigned)) != cudaSuccess ||
        cudaMalloc(&ctx->d_meta, (size_t)cfg->max_blocks * kBS3 * sizeof(unsigned short)) != cudaSuccess) {
        cudaGetLastError();
        return bail(GBFK_E_OOM);
    }
    cudaMemset(ctx->phi[0], 0, bytes);
    cudaMemset(ctx->phi[1], 0, bytes);
    cudaMemset(ctx->pw, 0, bytes);
    cudaMemset(ctx->pg, 0, bytes);
    cudaMemset(ctx->d_nan, 0, 2 * sizeof(unsigned));
    if (ensure_table(ctx) != GBFK_OK) return bail(GBFK_E_CUDA);
    *out = ctx;
    return GBFK_OK;
}

int gbfk_destroy(gbfk_ctx *ctx)
{
    if (!ctx) return GBFK_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    release_topology(ctx);
    void *ptrs[] = {ctx->phi[0], ctx->phi[1], ctx->pw, ctx->pg, ctx->d_nan, ctx->d_stage, ctx->d_ints, ctx->d_meta,
                    ctx->d_t1c, ctx->d_flair, ctx->d_pet, ctx->d_roi, ctx->d_model, ctx->d_partial, ctx->d_lik,
                    ctx->d_roi_count};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    for (void *p : ctx->adj_mem)
        if (p) cudaFree(p);
    if (ctx->io_ready) {
        cudaStreamSynchronize(ctx->io_in_stream);
        cudaStreamSynchronize(ctx->io_out_stream);
        for (int j = 0; j < 2; j++) {
            cudaFree(ctx->io_in[j]);
            cudaFree(ctx->io_out[j]);
            for (int k = 0; k < 4; k++) cudaEventDestroy(ctx->io_ev[k][j]);
        }
        cudaStreamDestroy(ctx->io_in_stream);
        cudaStreamDestroy(ctx->io_out_stream);
    }
    if (ctx->adj_fstream) {
        cudaStreamSynchronize(ctx->adj_fstream);
        cudaStreamDestroy(ctx->adj_fstream);
    }
    for (auto *m : {&ctx->adj_ev_write, &ctx->adj_ev_read})
        for (auto &kv : *m) cudaEventDestroy(kv.second);
    if (ctx->adj_ev_join) cudaEventDestroy(ctx->adj_ev_join);
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return GBFK_OK;
}

const char *gbfk_last_error(const gbfk_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int gbfk_join_copies(gbfk_ctx *ctx)
{
    if (!ctx) return GBFK_E_INVALID;
    if (ctx->io_calls == 0) return GBFK_OK;
    CK(cudaSetDevice(ctx->device));
    // the output stream runs its copies in order: its last event covers them all
    CK(cudaStreamWaitEvent(ctx->stream, ctx->io_ev[3][(ctx->io_calls - 1) & 1], 0));
    return GBFK_OK;
}

int gbfk_sync(gbfk_ctx *ctx)
{
    if (!ctx) return GBFK_E_INVALID;
    CK(cudaSetDevice(ctx->device));
    int rc = gbfk_join_copies(ctx);
    if (rc) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    return check_stage_timeout(ctx);
}

int gbfk_set_step_kernel(gbfk_ctx *ctx, int kind)
{
    if (!ctx) return GBFK_E_INVALID;
    if (kind != GBFK_STEP_AUTO && kind != GBFK_STEP_BLOCK && kind != GBFK_STEP_PIPELINED && kind != GBFK_STEP_RUN)
        return fail(ctx, GBFK_E_INVALID, "set_step_kernel: unknown kernel %d", kind);
    ctx->step_pref = kind;
    return GBFK_OK;
}

int gbfk_step_kernel(const gbfk_ctx *ctx) { return ctx ? ctx->step_used : 0; }

int64_t gbfk_launch_count(const gbfk_ctx *ctx) { return ctx ? ctx->launches : 0; }

int gbfk_num_blocks(const gbfk_ctx *ctx) { return ctx ? ctx->nblocks : 0; }

int gbfk_set_uniform(gbfk_ctx *ctx, int bpd)
{
    if (!ctx) return GBFK_E_INVALID;
    if (bpd <= 0 || (int64_t)bpd * bpd * bpd > ctx->max_blocks)
        return fail(ctx, GBFK_E_INVALID, "uniform grid of %d^3 blocks does not fit %d slots", bpd, ctx->max_blocks);
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->stream));
    free_topology(ctx);
    const int nb = bpd * bpd * bpd;
    ctx->nblocks = nb;
    ctx->bpd = bpd;
    ctx->uniform = true;
    ctx->h_slot.resize(nb);
    std::vector<int> nbr((size_t)nb * 6);
    for (int bz = 0; bz < bpd; bz++)
        for (int by = 0; by < bpd; by++)
            for (int bx = 0; bx < bpd; bx++) {
                const int b = bx + bpd * (by + bpd * bz);
                ctx->h_slot[b] = b;
                auto id = [&](int x, int y, int z) {
                    x = (x + bpd) % bpd; y = (y + bpd) % bpd; z = (z + bpd) % bpd;
                    return x + bpd * (y + bpd * z);
                };
                int *n = &nbr[(size_t)b * 6];
                n[0] = id(bx - 1, by, bz); n[1] = id(bx + 1, by, bz);
                n[2] = id(bx, by - 1, bz); n[3] = id(bx, by + 1, bz);
                n[4] = id(bx, by, bz - 1); n[5] = id(bx, by, bz + 1);
            }
    const double h = 1.0 / (8.0 * bpd);
    ctx->h_h.assign(nb, h);
    ctx->identity_slots = true;
    {
        int rc = topo_alloc(ctx, &ctx->d_slot, nb * sizeof(int));
        if (!rc) rc = topo_alloc(ctx, &ctx->d_nbr, (size_t)nb * 6 * sizeof(int));
        if (!rc) rc = topo_alloc(ctx, &ctx->d_h, nb * ctx->rsize);
        if (rc) return rc;
    }
    CK(cudaMemcpy(ctx->d_slot, ctx->h_slot.data(), nb * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->d_nbr, nbr.data(), (size_t)nb * 6 * sizeof(int), cudaMemcpyHostToDevice));
    if (ctx->precision == GBFK_F64) {
        std::vector<double> hv(nb, h);
        CK(cudaMemcpy(ctx->d_h, hv.data(), nb * sizeof(double), cudaMemcpyHostToDevice));
    } else {
        std::vector<float> hv(nb, (float)h);
        CK(cudaMemcpy(ctx->d_h, hv.data(), nb * sizeof(float), cudaMemcpyHostToDevice));
    }
    int rc = upload_ih2(ctx);
    if (rc) return rc;
    {
        int L = 0;
        while ((1 << L) < bpd) L++;
        std::vector<int> level(nb, L), index(3 * (size_t)nb);
        for (int b = 0; b < nb; b++) {
            index[3 * b] = b % bpd;
            index[3 * b + 1] = (b / bpd) % bpd;
            index[3 * b + 2] = b / (bpd * bpd);
        }
        if ((1 << L) == bpd) rc = upload_origin(ctx, level, index);
    }
    if (rc) return rc;
    ctx->have_topology = true;
    return GBFK_OK;
}

int gbfk_set_topology(gbfk_ctx *ctx, const gbfk_blockinfo *blocks, int nblocks, const gbfk_ghost_csr *g)
{
    if (!ctx) return GBFK_E_INVALID;
    if (!blocks || !g || nblocks <= 0) return fail(ctx, GBFK_E_INVALID, "set_topology: null or empty input");
    if (nblocks > ctx->max_blocks) return fail(ctx, GBFK_E_OOM, "set_topology: %d blocks > %d slots", nblocks, ctx->max_blocks);
    if (g->nrows != (int64_t)nblocks * kLabGhosts)
        return fail(ctx, GBFK_E_INVALID, "set_topology: %lld ghost rows, expected %d*488", (long long)g->nrows, nblocks);
    std::vector<char> used(ctx->max_blocks, 0);
    for (int i = 0; i < nblocks; i++) {
        const int s = blocks[i].slot;
        if (s < 0 || s >= ctx->max_blocks || used[s])
            return fail(ctx, GBFK_E_INVALID, "set_topology: bad or repeated slot %d", s);
        used[s] = 1;
    }
    const int64_t nnz = g->row_ptr[g->nrows];
    if (g->row_ptr[0] != 0 || nnz < 0) return fail(ctx, GBFK_E_INVALID, "set_topology: malformed row_ptr");
    std::vector<int> src(nnz);
    for (int64_t k = 0; k < nnz; k++) {
        const int64_t s = g->src[k];
        if (s < 0 || s >= (int64_t)ctx->max_blocks * kBS3 || !used[s / kBS3])
            return fail(ctx, GBFK_E_INVALID, "set_topology: ghost source %lld is not in a current block", (long long)s);
        src[k] = (int)s;
    }
    for (int64_t r = 0; r < g->nrows; r++)
        if (g->row_ptr[r + 1] < g->row_ptr[r]) return fail(ctx, GBFK_E_INVALID, "set_topology: row_ptr not monotone");
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->stream));
    free_topology(ctx);
    ctx->nblocks = nblocks;
    ctx->h_slot.resize(nblocks);
    ctx->h_h.resize(nblocks);
    ctx->identity_slots = true;
    for (int i = 0; i < nblocks; i++) {
        ctx->h_slot[i] = blocks[i].slot;
        ctx->h_h[i] = blocks[i].h;
        if (blocks[i].slot != i) ctx->identity_slots = false;
    }
    {
        int rc = topo_alloc(ctx, &ctx->d_slot, nblocks * sizeof(int));
        if (!rc) rc = topo_alloc(ctx, &ctx->d_h, nblocks * ctx->rsize);
        if (rc) return rc;
    }
    CK(cudaMemcpy(ctx->d_slot, ctx->h_slot.data(), nblocks * sizeof(int), cudaMemcpyHostToDevice));
    if (ctx->precision == GBFK_F64) {
        CK(cudaMemcpy(ctx->d_h, ctx->h_h.data(), nblocks * sizeof(double), cudaMemcpyHostToDevice));
    } else {
        std::vector<float> hv(nblocks);
        for (int i = 0; i < nblocks; i++) hv[i] = (float)ctx->h_h[i];
        CK(cudaMemcpy(ctx->d_h, hv.data(), nblocks * sizeof(float), cudaMemcpyHostToDevice));
    }
    int rc = ctx->precision == GBFK_F64 ? set_csr<double>(ctx, g->row_ptr, src, g->w0, g->w1, g->w2, true)
                                        : set_csr<float>(ctx, g->row_ptr, src, g->w0, g->w1, g->w2, true);
    if (rc) return rc;
    rc = upload_ih2(ctx);
    if (rc) return rc;
    {
        std::vector<int> level(nblocks), index(3 * (size_t)nblocks);
        for (int i = 0; i < nblocks; i++) {
            level[i] = blocks[i].level;
            for (int d = 0; d < 3; d++) index[3 * i + d] = blocks[i].index[d];
        }
        rc = upload_origin(ctx, level, index);
        if (rc) return rc;
    }
    ctx->have_topology = true;
    return GBFK_OK;
}

int gbfk_upload_field(gbfk_ctx *ctx, int field, const void *host, int64_t first, int64_t ncells)
{
    if (!ctx) return GBFK_E_INVALID;
    if (field == GBFK_PHI) ctx->phi_clamped = false;
    void *p = field_ptr(ctx, field);
    if (!p || !host || first < 0 || ncells < 0 || first + ncells > (int64_t)ctx->max_blocks * kBS3)
        return fail(ctx, GBFK_E_INVALID, "upload_field: bad field or range");
    CK(cudaSetDevice(ctx->device));
    CK(cudaMemcpyAsync((char *)p + first * ctx->rsize, host, ncells * ctx->rsize, cudaMemcpyHostToDevice,
                       ctx->stream));
    if (field != GBFK_PHI) invalidate_static(ctx);
    return GBFK_OK;
}

int gbfk_download_field(gbfk_ctx *ctx, int field, void *host, int64_t first, int64_t ncells)
{
    if (!ctx) return GBFK_E_INVALID;
    void *p = field_ptr(ctx, field);
    if (!p || !host || first < 0 || ncells < 0 || first + ncells > (int64_t)ctx->max_blocks * kBS3)
        return fail(ctx, GBFK_E_INVALID, "download_field: bad field or range");
    CK(cudaSetDevice(ctx->device));
    CK(cudaMemcpyAsync(host, (const char *)p + first * ctx->rsize, ncells * ctx->rsize, cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return GBFK_OK;
}

static int dense_io(gbfk_ctx *ctx, int field, void *host, int n, bool up)
{
    if (!ctx) return GBFK_E_INVALID;
    if (!ctx->uniform || n != 8 * ctx->bpd)
        return fail(ctx, GBFK_E_STATE, "dense transfer needs a uniform topology with n = 8*bpd");
    void *p = field_ptr(ctx, field);
    if (!p || !host) return fail(ctx, GBFK_E_INVALID, "dense transfer: bad field or buffer");
    CK(cudaSetDevice(ctx->device));
    const size_t bytes = (size_t)n * n * n * ctx->rsize;
    if (ctx->stage_bytes < bytes) {
        if (ctx->d_stage) cudaFree(ctx->d_stage);
        ctx->d_stage = nullptr;
        ctx->stage_bytes = 0;
        CK(cudaMalloc(&ctx->d_stage, bytes));
        ctx->stage_bytes = bytes;
    }
    if (up) {
        CK(cudaMemcpyAsync(ctx->d_stage, host, bytes, cudaMemcpyHostToDevice, ctx->stream));
        if (ctx->precision == GBFK_F64)
            CK(launch_dense_scatter<double>((const double *)ctx->d_stage, (double *)p, n, true, ctx->stream));
        else
            CK(launch_dense_scatter<float>((const float *)ctx->d_stage, (float *)p, n, true, ctx->stream));
        ctx->launches++;
        if (field != GBFK_PHI) invalidate_static(ctx);
    } else {
        if (ctx->precision == GBFK_F64)
            CK(launch_dense_scatter<double>((const double *)p, (double *)ctx->d_stage, n, false, ctx->stream));
        else
            CK(launch_dense_scatter<float>((const float *)p, (float *)ctx->d_stage, n, false, ctx->stream));
        ctx->launches++;
        CK(cudaMemcpyAsync(host, ctx->d_stage, bytes, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    return GBFK_OK;
}

int gbfk_upload_dense(gbfk_ctx *ctx, int field, const void *host, int n)
{
    if (ctx && field == GBFK_PHI) ctx->phi_clamped = false;
    return dense_io(ctx, field, const_cast<void *>(host), n, true);
}

int gbfk_download_dense(gbfk_ctx *ctx, int field, void *host, int n) { return dense_io(ctx, field, host, n, false); }

int gbfk_rd_step_host(gbfk_ctx *ctx, const void *host_in, void *host_out, double Dw, double Dg, double rho,
                      double dt, int nsteps)
{
    if (!ctx) return GBFK_E_INVALID;
    if (!ctx->have_topology || !ctx->uniform) return fail(ctx, GBFK_E_STATE, "rd_step_host: needs a uniform grid");
    if (!host_in || !host_out || nsteps < 0) return fail(ctx, GBFK_E_INVALID, "rd_step_host: bad arguments");
    CK(cudaSetDevice(ctx->device));
    const int n = 8 * ctx->bpd;
    const size_t bytes = (size_t)n * n * n * ctx->rsize;
    if (!ctx->io_ready || ctx->io_bytes < bytes) {
        if (ctx->io_ready) {
            CK(cudaStreamSynchronize(ctx->io_in_stream));
            CK(cudaStreamSynchronize(ctx->io_out_stream));
            CK(cudaStreamSynchronize(ctx->stream));
            for (int j = 0; j < 2; j++) {
                cudaFree(ctx->io_in[j]);
                cudaFree(ctx->io_out[j]);
                ctx->io_in[j] = ctx->io_out[j] = nullptr;
            }
        } else {
            CK(cudaStreamCreateWithFlags(&ctx->io_in_stream, cudaStreamNonBlocking));
            CK(cudaStreamCreateWithFlags(&ctx->io_out_stream, cudaStreamNonBlocking));
            for (int j = 0; j < 2; j++)
                for (int k = 0; k < 4; k++) CK(cudaEventCreateWithFlags(&ctx->io_ev[k][j], cudaEventDisableTiming));
            ctx->io_ready = true;
        }
        ctx->io_bytes = 0;
        ctx->io_calls = 0;
        for (int j = 0; j < 2; j++) {
            CK(cudaMalloc(&ctx->io_in[j], bytes));
            CK(cudaMalloc(&ctx->io_out[j], bytes));
        }
        ctx->io_bytes = bytes;
    }
    const int j = (int)(ctx->io_calls & 1);
    cudaEvent_t *ev_in_ready = ctx->io_ev[0], *ev_in_free = ctx->io_ev[1], *ev_out_ready = ctx->io_ev[2],
                *ev_out_free = ctx->io_ev[3];
    // input: H2D on the input stream once call k - 2 has scattered this staging buffer
    if (ctx->io_calls >= 2) CK(cudaStreamWaitEvent(ctx->io_in_stream, ev_in_free[j], 0));
    CK(cudaMemcpyAsync(ctx->io_in[j], host_in, bytes, cudaMemcpyHostToDevice, ctx->io_in_stream));
    CK(cudaEventRecord(ev_in_ready[j], ctx->io_in_stream));
    // the context's stream: scatter into the blocks, the steps, gather
    CK(cudaStreamWaitEvent(ctx->stream, ev_in_ready[j], 0));
    void *phi = field_ptr(ctx, GBFK_PHI);
    if (ctx->precision == GBFK_F64)
        CK(launch_dense_scatter<double>((const double *)ctx->io_in[j], (double *)phi, n, true, ctx->stream));
    else
        CK(launch_dense_scatter<float>((const float *)ctx->io_in[j], (float *)phi, n, true, ctx->stream));
    CK(cudaEventRecord(ev_in_free[j], ctx->stream));
    ctx->launches++;
    ctx->phi_clamped = false;
    const int rc = ctx->precision == GBFK_F64 ? rd_step_impl<double>(ctx, Dw, Dg, rho, dt, nsteps, 0)
                                              : rd_step_impl<float>(ctx, Dw, Dg, rho, dt, nsteps, 0);
    if (rc) return rc;
    if (ctx->io_calls >= 2) CK(cudaStreamWaitEvent(ctx->stream, ev_out_free[j], 0));
    phi = field_ptr(ctx, GBFK_PHI);
    if (ctx->precision == GBFK_F64)
        CK(launch_dense_scatter<double>((const double *)phi, (double *)ctx->io_out[j], n, false, ctx->stream));
    else
        CK(launch_dense_scatter<float>((const float *)phi, (float *)ctx->io_out[j], n, false, ctx->stream));
    CK(cudaEventRecord(ev_out_ready[j], ctx->stream));
    ctx->launches++;
    // output: D2H on the output stream, overlapping the next call's input copy
    CK(cudaStreamWaitEvent(ctx->io_out_stream, ev_out_ready[j], 0));
    CK(cudaMemcpyAsync(host_out, ctx->io_out[j], bytes, cudaMemcpyDeviceToHost, ctx->io_out_stream));
    CK(cudaEventRecord(ev_out_free[j], ctx->io_out_stream));
    ctx->io_calls++;
    return GBFK_OK;
}

int gbfk_rd_step(gbfk_ctx *ctx, double Dw, double Dg, double rho, double dt, int nsteps, int check_nan)
{
    if (!ctx) return GBFK_E_INVALID;
    if (!ctx->have_topology) return fail(ctx, GBFK_E_STATE, "rd_step: no topology");
    if (nsteps < 0) return fail(ctx, GBFK_E_INVALID, "rd_step: negative step count");
    CK(cudaSetDevice(ctx->device));
    return ctx->precision == GBFK_F64 ? rd_step_impl<double>(ctx, Dw, Dg, rho, dt, nsteps, check_nan)
                                      : rd_step_impl<float>(ctx, Dw, Dg, rho, dt, nsteps, check_nan);
}

int gbfk_rd_rhs(gbfk_ctx *ctx, double Dw, double Dg, double rho, void *host)
{
    if (!ctx) return GBFK_E_INVALID;
    if (!ctx->have_topology) return fail(ctx, GBFK_E_STATE, "rd_rhs: no topology");
    if (!host) return fail(ctx, GBFK_E_INVALID, "rd_rhs: null output");
    CK(cudaSetDevice(ctx->device));
    return ctx->precision == GBFK_F64 ? rd_rhs_impl<double>(ctx, Dw, Dg, rho, host)
                                      : rd_rhs_impl<float>(ctx, Dw, Dg, rho, host);
}

}  // extern "C"

template <typename Real>
static int cfl_impl(gbfk_ctx *ctx, double Dw, double Dg, double *out)
{
    const int nparts = 148 * 4;
    if (!ctx->d_partial) CK(cudaMalloc(&ctx->d_partial, (size_t)148 * 4 * 7 * sizeof(double)));
    const Real dw = (Real)Dw, dg = (Real)Dg;
    CK(launch_cfl<Real>(view<Real>(ctx), dw, dg, ctx->d_partial, nparts, ctx->stream));
    ctx->launches++;
    std::vector<double> part(2 * (size_t)nparts);
    CK(cudaMemcpyAsync(part.data(), ctx->d_partial, part.size() * sizeof(double), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    double dmax = 0, hmin = INFINITY;
    for (int i = 0; i < nparts; i++) {
        dmax = std::fmax(dmax, part[2 * i]);
        hmin = std::fmin(hmin, part[2 * i + 1]);
    }
    // Glioma_ReactionDiffusion.cpp:306-307 in Real, with h the finest leaf's
    const Real h = (Real)hmin;
    const Real mx = dw >= dg ? dw : dg;
    out[0] = (double)(Real)(0.99 * (double)h * (double)h / (2. * 3 * (double)mx));
    out[1] = hmin;
    out[2] = dmax;
    return GBFK_OK;
}

extern "C" {

int gbfk_cfl(gbfk_ctx *ctx, double Dw, double Dg, double out[3])
{
    if (!ctx) return GBFK_E_INVALID;
    if (!ctx->have_topology) return fail(ctx, GBFK_E_STATE, "cfl: no topology");
    if (!out) return fail(ctx, GBFK_E_INVALID, "cfl: null output");
    CK(cudaSetDevice(ctx->device));
    return ctx->precision == GBFK_F64 ? cfl_impl<double>(ctx, Dw, Dg, out) : cfl_impl<float>(ctx, Dw, Dg, out);
}

int gbfk_fwt_details(gbfk_ctx *ctx, double *out)
{
    if (!ctx) return GBFK_E_INVALID;
    if (!ctx->have_topology) return fail(ctx, GBFK_E_STATE, "fwt_details: no topology");
    if (!out) return fail(ctx, GBFK_E_INVALID, "fwt_details: null output");
    CK(cudaSetDevice(ctx->device));
    return ctx->precision == GBFK_F64 ? fwt_impl<double>(ctx, out) : fwt_impl<float>(ctx, out);
}

int gbfk_split(gbfk_ctx *ctx, int nsplit, const int *parents, const int *children)
{
    if (!ctx) return GBFK_E_INVALID;
    if (!ctx->have_topology) return fail(ctx, GBFK_E_STATE, "split: no topology");
    if (nsplit < 0 || (nsplit && (!parents || !children))) return fail(ctx, GBFK_E_INVALID, "split: bad arguments");
    if (nsplit == 0) return GBFK_OK;
    CK(cudaSetDevice(ctx->device));
    return ctx->precision == GBFK_F64 ? split_impl<double>(ctx, nsplit, parents, children)
                                      : split_impl<float>(ctx, nsplit, parents, children);
}

int gbfk_collapse(gbfk_ctx *ctx, int n, const int *children, const int *parents)
{
    if (!ctx) return GBFK_E_INVALID;
    if (n < 0 || (n && (!parents || !children))) return fail(ctx, GBFK_E_INVALID, "collapse: bad arguments");
    if (n == 0) return GBFK_OK;
    CK(cudaSetDevice(ctx->device));
    return ctx->precision == GBFK_F64 ? collapse_impl<double>(ctx, n, children, parents)
                                      : collapse_impl<float>(ctx, n, children, parents);
}

static int dump_to_device(gbfk_ctx *ctx, int n)
{
    if (!ctx->have_topology) return fail(ctx, GBFK_E_STATE, "uq_dump: no topology");
    if (!ctx->have_origin) return fail(ctx, GBFK_E_STATE, "uq_dump: block origins unknown (non power-of-two uniform grid)");
    if (n <= 0 || (int64_t)n * n * n > ((int64_t)1 << 34)) return fail(ctx, GBFK_E_INVALID, "uq_dump: bad grid size %d", n);
    const size_t bytes = (size_t)n * n * n * sizeof(double);
    if (ctx->model_bytes < bytes) {
        if (ctx->d_model) cudaFree(ctx->d_model);
        ctx->d_model = nullptr;
        ctx->model_bytes = 0;
        CK(cudaMalloc(&ctx->d_model, bytes));
        ctx->model_bytes = bytes;
    }
    if (ctx->precision == GBFK_F64)
        CK(launch_uq_dump<double>(ctx->d_slot, (const double *)ctx->d_origin, (const double *)ctx->d_h, ctx->nblocks,
                                  (const double *)ctx->phi[ctx->cur], n, ctx->d_model, ctx->stream));
    else
        CK(launch_uq_dump<float>(ctx->d_slot, (const float *)ctx->d_origin, (const float *)ctx->d_h, ctx->nblocks,
                                 (const float *)ctx->phi[ctx->cur], n, ctx->d_model, ctx->stream));
    ctx->launches++;
    return GBFK_OK;
}

int gbfk_uq_dump(gbfk_ctx *ctx, int n, double *host_out)
{
    if (!ctx) return GBFK_E_INVALID;
    if (!host_out) return fail(ctx, GBFK_E_INVALID, "uq_dump: null output");
    CK(cudaSetDevice(ctx->device));
    int rc = dump_to_device(ctx, n);
    if (rc) return rc;
    CK(cudaMemcpyAsync(host_out, ctx->d_model, (size_t)n * n * n * sizeof(double), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return GBFK_OK;
}

int gbfk_set_observations(gbfk_ctx *ctx, int n, const double *t1c, const double *flair, const double *pet,
                          const int *roi, int nroi)
{
    if (!ctx) return GBFK_E_INVALID;
    if (n <= 0 || !t1c || !flair || nroi < 0 || (nroi > 0 && !roi))
        return fail(ctx, GBFK_E_INVALID, "set_observations: bad arguments");
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->stream));
    void *old[] = {ctx->d_t1c, ctx->d_flair, ctx->d_pet, ctx->d_roi};
    for (void *p : old)
        if (p) cudaFree(p);
    ctx->d_t1c = ctx->d_flair = nullptr;
    ctx->d_pet = nullptr;
    ctx->d_roi = nullptr;
    const size_t N = (size_t)n * n * n;
    std::vector<unsigned char> a(N), b(N);
    for (size_t i = 0; i < N; i++) {
        a[i] = t1c[i] == 1 ? 1 : 0;
        b[i] = flair[i] == 1 ? 1 : 0;
    }
    CK(cudaMalloc(&ctx->d_t1c, N));
    CK(cudaMalloc(&ctx->d_flair, N));
    CK(cudaMemcpy(ctx->d_t1c, a.data(), N, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->d_flair, b.data(), N, cudaMemcpyHostToDevice));
    if (pet) {
        CK(cudaMalloc(&ctx->d_pet, N * sizeof(double)));
        CK(cudaMemcpy(ctx->d_pet, pet, N * sizeof(double), cudaMemcpyHostToDevice));
    }
    if (roi && nroi > 0) {
        for (int i = 0; i < 3 * nroi; i++)
            if (roi[i] < 0 || roi[i] >= n) return fail(ctx, GBFK_E_INVALID, "set_observations: ROI point out of the grid");
        CK(cudaMalloc(&ctx->d_roi, (size_t)nroi * 3 * sizeof(int)));
        CK(cudaMemcpy(ctx->d_roi, roi, (size_t)nroi * 3 * sizeof(int), cudaMemcpyHostToDevice));
    }
    ctx->nroi = roi ? nroi : 0;
    ctx->obs_n = n;
    return GBFK_OK;
}

int gbfk_log_likelihood(gbfk_ctx *ctx, const gbfk_likelihood_params *p, double out[4])
{
    if (!ctx) return GBFK_E_INVALID;
    if (!p || !out) return fail(ctx, GBFK_E_INVALID, "log_likelihood: null argument");
    if (!ctx->obs_n) return fail(ctx, GBFK_E_STATE, "log_likelihood: no observations");
    if (p->step_pet <= 0 || p->step_mri <= 0 || !(p->slope != 0))
        return fail(ctx, GBFK_E_INVALID, "log_likelihood: bad parameters");
    CK(cudaSetDevice(ctx->device));
    int rc = dump_to_device(ctx, ctx->obs_n);
    if (rc) return rc;
    const int nparts = 148 * 4;
    if (!ctx->d_partial) CK(cudaMalloc(&ctx->d_partial, (size_t)nparts * 7 * sizeof(double)));
    if (!ctx->d_lik) CK(cudaMalloc(&ctx->d_lik, 4 * sizeof(double)));
    LikelihoodParams lp;
    lp.pet_sigma2 = p->pet_sigma2;
    lp.pet_scale = p->pet_scale;
    lp.t1_uc = p->t1_uc;
    lp.t2_uc = p->t2_uc;
    lp.slope = p->slope;
    lp.step_pet = p->step_pet;
    lp.step_mri = p->step_mri;
    CK(launch_likelihood(ctx->d_model, ctx->obs_n, ctx->d_t1c, ctx->d_flair, ctx->d_pet,
                         ctx->nroi ? ctx->d_roi : nullptr, ctx->nroi, lp, ctx->d_partial, nparts, ctx->d_lik,
                         ctx->stream));
    ctx->launches += 2;
    CK(cudaMemcpyAsync(out, ctx->d_lik, 4 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return GBFK_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Forward + discrete adjoint with binomial checkpointing.
namespace {

template <typename Real>
struct Adjoint {
    gbfk_ctx *ctx;
    PoolView<Real> v;
    size_t fbytes;
    Real *T0, *T1, *T2, *LAM;
    std::vector<Real *> slots;
    double *grad_acc;
    bool abs_terms = false;  // also sum the magnitudes of the gradient terms
    // the blocks the adjoint steps run (NULL: all): every block that can hold
    // a domain cell, and their face neighbours
    const int *blocks = nullptr;
    int nlaunch = 0;
    Real rho;
    double dt, Dw;
    int64_t fsteps = 0, asteps = 0;
    cudaError_t err = cudaSuccess;
    // forward steps on the pipelined kernel: its work lists, 1/(h*h) of the
    // uniform grid, and the face-box tensor maps of every buffer a step reads
    bool pipelined = false;
    BlockLists lists{};
    double ih2 = 0;
    const Real *X0 = nullptr;  // the initial condition: the only step input not written by a step
    struct Maps {
        const void *buf;
        CUtensorMap m[3];
    };
    std::vector<Maps> maps;
    std::unordered_map<const void *, size_t> map_index;

    cudaError_t add_maps(const void *buf)
    {
        maps.emplace_back();
        maps.back().buf = buf;
        map_index[buf] = maps.size() - 1;
        return make_pool_tensor_maps(const_cast<void *>(buf), ctx->max_blocks, (int)sizeof(Real), maps.back().m);
    }
    const CUtensorMap *maps_of(const void *buf) const
    {
        const auto it = map_index.find(buf);
        return it == map_index.end() ? nullptr : maps[it->second].m;
    }

    // skip_empty: every empty block of the initial condition holds +0 (and
    // dt is finite), so every step writes +0 there; a step then runs only the
    // heavy blocks when its output buffer's empty blocks already hold +0
    // (ctx->adj_clean), which every full step into a buffer establishes
    bool skip_empty = false;
    bool clean(const void *b) const { return skip_empty && (b == X0 || ctx->adj_clean.count(b) != 0); }

    // Two streams: forward steps on fs, adjoint steps on ctx->stream, so that
    // the recomputation of the states ahead can overlap the adjoint steps
    // (both are latency-bound on small grids).  The only buffers both touch
    // are the states the adjoint steps read: an adjoint step waits for the
    // forward write of its state, a forward write waits for the adjoint reads
    // before it (one event per buffer and kind, re-recorded; a wait binds the
    // record before it).  fs == ctx->stream runs everything in one stream.
    cudaStream_t fs = nullptr;
    std::unordered_set<const void *> wait_write, wait_read;  // records not yet waited for
    cudaEvent_t event_of(std::unordered_map<const void *, cudaEvent_t> &m, const void *b)
    {
        auto it = m.find(b);
        if (it != m.end()) return it->second;
        cudaEvent_t e = nullptr;
        if (err == cudaSuccess) err = cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
        if (err != cudaSuccess) return nullptr;
        m[b] = e;
        return e;
    }
    void forward_writes(const void *dst)  // before a forward op writes dst
    {
        if (fs == ctx->stream || err != cudaSuccess || !wait_read.erase(dst)) return;
        cudaEvent_t e = event_of(ctx->adj_ev_read, dst);
        if (e) err = cudaStreamWaitEvent(fs, e, 0);
    }
    void forward_wrote(const void *dst)
    {
        if (fs == ctx->stream || err != cudaSuccess) return;
        cudaEvent_t e = event_of(ctx->adj_ev_write, dst);
        if (e) err = cudaEventRecord(e, fs);
        wait_write.insert(dst);
    }
    void adjoint_reads(const void *b)  // before an op on ctx->stream reads b
    {
        if (fs == ctx->stream || err != cudaSuccess || !wait_write.erase(b)) return;
        cudaEvent_t e = event_of(ctx->adj_ev_write, b);
        if (e) err = cudaStreamWaitEvent(ctx->stream, e, 0);
    }
    void adjoint_read(const void *b)
    {
        if (fs == ctx->stream || err != cudaSuccess) return;
        cudaEvent_t e = event_of(ctx->adj_ev_read, b);
        if (e) err = cudaEventRecord(e, ctx->stream);
        wait_read.insert(b);
    }
    // `to` waits for everything enqueued on `from` so far
    void join(cudaStream_t from, cudaStream_t to)
    {
        if (from == to || err != cudaSuccess) return;
        if (!ctx->adj_ev_join) err = cudaEventCreateWithFlags(&ctx->adj_ev_join, cudaEventDisableTiming);
        if (err == cudaSuccess) err = cudaEventRecord(ctx->adj_ev_join, from);
        if (err == cudaSuccess) err = cudaStreamWaitEvent(to, ctx->adj_ev_join, 0);
    }

    void step(const Real *in, Real *out)
    {
        if (err != cudaSuccess) return;
        const CUtensorMap *m = pipelined ? maps_of(in) : nullptr;
        if (m) {
            const bool skip = skip_empty && clean(in) && clean(out);
            err = launch_rd_step_tma<Real>(v, lists, (const Real *)ctx->d_H, ctx->d_meta, ih2, in, in != X0, out, rho,
                                           dt, ctx->d_nan, ctx->d_nan + 1, m, skip, fs);
            if (skip_empty) ctx->adj_clean.insert(out);
        } else
            err = launch_rd_step<Real>(v, (const Real *)ctx->d_H, ctx->d_meta, ctx->d_ih2, in, out, nullptr, rho, dt,
                                       ctx->d_nan, fs);
        fsteps++;
        ctx->launches++;
    }
    // k forward steps from src into dst; intermediate states alternate
    // between T0 and T1 (src and dst are never T0/T1 and never equal)
    void advance(const Real *src, Real *dst, int k)
    {
        if (err != cudaSuccess) return;
        if (k == 0) {
            if (src != dst) {
                forward_writes(dst);
                if (err == cudaSuccess) err = cudaMemcpyAsync(dst, src, fbytes, cudaMemcpyDeviceToDevice, fs);
                if (clean(src)) ctx->adj_clean.insert(dst);
                else ctx->adj_clean.erase(dst);
                forward_wrote(dst);
            }
            return;
        }
        forward_writes(dst);
        const Real *cur = src;
        for (int s = 0; s < k; s++) {
            Real *out = (s == k - 1) ? dst : (cur == T0 ? T1 : T0);
            step(cur, out);
            cur = out;
        }
        forward_wrote(dst);
    }
    // The checkpoint buffers the schedule may fill, first in, first out (the
    // buffer released longest ago, whose adjoint reads are most likely done).
    // The schedule never holds more than the checkpoint count.
    std::deque<Real *> free_slots;
    Real *take_slot()
    {
        if (free_slots.empty()) {
            if (err == cudaSuccess) err = cudaErrorInvalidValue;
            return T2;
        }
        Real *s = free_slots.front();
        free_slots.pop_front();
        return s;
    }
    void release_slot(Real *s) { free_slots.push_back(s); }
    // the adjoint state between launches (double-buffered); `latest` is the
    // set the last launch wrote
    AdjBuffers sets[2];
    int latest = 0;
    // one adjoint step through the forward step from phi_k (one launch)
    void adjoint_step(const Real *phi_k)
    {
        if (err != cudaSuccess) return;
        adjoint_reads(phi_k);
        if (err != cudaSuccess) return;
        err = launch_adjoint_fused<Real>(v, (const Real *)ctx->d_H, ctx->d_meta, ctx->d_ih2, phi_k, LAM, sets[latest],
                                         sets[latest ^ 1], asteps == 0 ? 1 : 0, abs_terms, blocks, nlaunch, rho, dt,
                                         Dw, grad_acc, ctx->stream);
        adjoint_read(phi_k);
        latest ^= 1;
        ctx->launches++;
        asteps++;
    }
    // lambda_0 into LAM after the sweep (LAM already holds it when no step ran)
    void finish()
    {
        if (err != cudaSuccess || asteps == 0) return;
        // the blocks that are not run hold lambda_0 = 0
        if (blocks) err = cudaMemsetAsync(LAM, 0, fbytes, ctx->stream);
        if (err != cudaSuccess) return;
        err = launch_adjoint_fused<Real>(v, (const Real *)ctx->d_H, ctx->d_meta, ctx->d_ih2, nullptr, LAM,
                                         sets[latest], sets[latest ^ 1], 2, false, blocks, nlaunch, rho, dt, Dw,
                                         grad_acc, ctx->stream);
        ctx->launches++;
    }
    static double beta(int c, int r)  // C(c + r, c) = C(c + r, r), capped; 0 for r < 0
    {
        if (r < 0) return 0;
        const int k = std::min(c, r), m = std::max(c, r);
        double b = 1;
        for (int i = 1; i <= k; i++) {
            b = b * (m + i) / i;
            if (b > 1e18) return 1e18;
        }
        return b;
    }
    // Binomial checkpointing (Griewank and Walther, "Algorithm 799: revolve",
    // ACM TOMS 26(1), 2000): reversing l steps from a stored state with c free
    // buffers costs the fewest forward steps when the first checkpoint goes
    // l1 steps ahead, l1 in [max(b(s, r-2), l - b(s-1, r)),
    // min(b(s, r-1), l - b(s-1, r-1))], with s = c + 1 states held (the
    // start's own buffer counts) and r the smallest repetition number with
    // b(s, r) >= l, b(s, r) = C(s + r, s).  Inside the recursion the lower end
    // is taken; on the chain of checkpoints that the first forward sweep
    // stores on its way to the horizon, the upper end (those states cost no
    // extra steps there).
    static int split(int l, int c, bool upper)
    {
        const int s = c + 1;
        int r = 0;
        while (beta(s, r) < l) r++;
        const double lo = std::max(beta(s, r - 2), l - beta(s - 1, r));
        const double hi = std::min(beta(s, r - 1), l - beta(s - 1, r - 1));
        const double pick = upper ? std::max(lo, hi) : lo;
        return (int)std::max(1.0, std::min(pick, (double)(l - 1)));
    }
    // The first forward sweep from X (phi_0) to the horizon state F, storing
    // the states at the chain positions a + split(l, c, true) in slots[c-1],
    // slots[c-2], ... (the states reverse_chain expects there).
    void sweep(const Real *X, Real *F, int nsteps, int c)
    {
        int pos = 0;
        const Real *cur = X;
        while (nsteps - pos > 1 && c > 0 && err == cudaSuccess) {
            const int l1 = split(nsteps - pos, c, true);
            advance(cur, slots[c - 1], l1);
            cur = slots[c - 1];
            pos += l1;
            c--;
        }
        advance(cur, F, nsteps - pos);
        free_slots.assign(slots.begin(), slots.begin() + c);
    }
    // reverse() along the chain stored by sweep(): slots[c-1] already holds
    // the state a + split(b - a, c, true); that buffer is free once the part
    // of the chain after it is reversed.
    void reverse_chain(int a, int b, int c, Real *X)
    {
        const int l = b - a;
        if (l <= 1 || c == 0 || err != cudaSuccess) {
            reverse(a, b, c, X);
            return;
        }
        const int l1 = split(l, c, true);
        Real *S = slots[c - 1];
        reverse_chain(a + l1, b, c - 1, S);
        release_slot(S);
        reverse(a, a + l1, c, X);
    }
    // X holds phi_a; LAM holds dL/dphi_b on entry and dL/dphi_a on exit;
    // c checkpoint buffers are free.
    void reverse(int a, int b, int c, Real *X)
    {
        const int l = b - a;
        if (l <= 0 || err != cudaSuccess) return;
        if (l == 1) {
            adjoint_step(X);
            return;
        }
        if (c == 0) {
            for (int k = b - 1; k > a; k--) {
                advance(X, T2, k - a);
                adjoint_step(T2);
            }
            adjoint_step(X);
            return;
        }
        const int l1 = split(l, c, false);
        Real *S = take_slot();
        advance(X, S, l1);
        reverse(a + l1, b, c - 1, S);
        release_slot(S);
        reverse(a, a + l1, c, X);
    }
};

template <typename Real>
int forward_adjoint_impl(gbfk_ctx *ctx, const gbfk_adjoint_params *p, gbfk_adjoint_result *res, void *grad_c0)
{
    int rc = prepare_static<Real>(ctx, p->Dw, p->Dg);
    if (rc) return rc;
    const int nb = ctx->nblocks, bpd = ctx->bpd, n = 8 * bpd;
    Adjoint<Real> A;
    A.ctx = ctx;
    A.v = view<Real>(ctx);
    A.fbytes = (size_t)nb * kBS3 * sizeof(Real);
    A.rho = (Real)p->rho;
    A.dt = p->dt;
    A.Dw = (double)(Real)p->Dw;
    // buffers: X0, F, T0, T1, T2, LAM, mu and cell flags + block status of
    // adjoint set 0, gradient partials, x0-gradient partials, the
    // checkpoints, then mu and flags of set 1 and the self terms of both
    // sets; kept in the context between calls
    const int xparts = 148 * 4;
    const size_t selfbytes = (size_t)nb * kBS3 * sizeof(double);
    const size_t sizes[16] = {A.fbytes, A.fbytes, A.fbytes, A.fbytes, A.fbytes, A.fbytes, A.fbytes,
                              (size_t)nb * kAdjFlagBytesPerBlock, (size_t)nb * kGradSlots * sizeof(double),
                              (size_t)xparts * 6 * sizeof(double), 0, A.fbytes,
                              (size_t)nb * kAdjFlagBytesPerBlock, selfbytes, selfbytes,
                              (size_t)nb * (sizeof(int) + 1)};
    auto release = [&]() {
        cudaStreamSynchronize(ctx->stream);
        if (ctx->adj_fstream) cudaStreamSynchronize(ctx->adj_fstream);
        // the per-buffer events belong to the buffers being freed
        for (auto *m : {&ctx->adj_ev_write, &ctx->adj_ev_read}) {
            for (auto &kv : *m) cudaEventDestroy(kv.second);
            m->clear();
        }
        for (void *q : ctx->adj_mem)
            if (q) cudaFree(q);
        ctx->adj_mem.clear();
        ctx->adj_fbytes = 0;
        ctx->adj_nblocks = ctx->adj_nsnap = 0;
        ctx->adj_clean.clear();
    };
    cudaError_t e = cudaSuccess;
    bool fresh = false;  // buffers allocated (and zeroed) by this call
    if (ctx->adj_fbytes != A.fbytes || ctx->adj_nblocks != nb || ctx->adj_nsnap < p->nsnapshots) {
        release();
        // the work fields one by one, the checkpoints in one allocation
        ctx->adj_mem.assign(16, nullptr);
        for (size_t i = 0; i < 16 && e == cudaSuccess; i++)
            e = cudaMalloc(&ctx->adj_mem[i], i != 10 ? sizes[i] : A.fbytes * (size_t)p->nsnapshots);
        if (e != cudaSuccess) {
            cudaGetLastError();
            release();
            return fail(ctx, GBFK_E_OOM, "forward_adjoint: %s", cudaGetErrorString(e));
        }
        ctx->adj_fbytes = A.fbytes;
        ctx->adj_nblocks = nb;
        ctx->adj_nsnap = p->nsnapshots;
        // the forward states start at +0 everywhere: every later step into
        // them may skip the empty blocks (see Adjoint::skip_empty)
        for (int i : {0, 1, 2, 3, 4})
            if (e == cudaSuccess) e = cudaMemsetAsync(ctx->adj_mem[i], 0, A.fbytes, ctx->stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(ctx->adj_mem[10], 0, A.fbytes * (size_t)p->nsnapshots, ctx->stream);
        if (e != cudaSuccess) {
            release();
            return fail(ctx, GBFK_E_CUDA, "forward_adjoint: %s", cudaGetErrorString(e));
        }
        fresh = true;
    }
    auto cleanup = [&]() {
        cudaStreamSynchronize(ctx->stream);
        if (ctx->adj_fstream) cudaStreamSynchronize(ctx->adj_fstream);
    };
    // the forward steps' own stream (GBFK_ADJ_STREAMS=1: everything on ctx->stream)
    A.fs = ctx->stream;
    if (const char *s = getenv("GBFK_ADJ_STREAMS"); !(s && atoi(s) == 1)) {
        if (!ctx->adj_fstream) e = cudaStreamCreateWithFlags(&ctx->adj_fstream, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            ctx->adj_fstream = nullptr;
            return fail(ctx, GBFK_E_CUDA, "forward_adjoint: %s", cudaGetErrorString(e));
        }
        A.fs = ctx->adj_fstream;
    }
    Real *X0 = (Real *)ctx->adj_mem[0], *F = (Real *)ctx->adj_mem[1];
    A.T0 = (Real *)ctx->adj_mem[2];
    A.T1 = (Real *)ctx->adj_mem[3];
    A.T2 = (Real *)ctx->adj_mem[4];
    A.LAM = (Real *)ctx->adj_mem[5];
    A.grad_acc = (double *)ctx->adj_mem[8];
    for (int k = 0; k < 2; k++) {
        unsigned char *fl = (unsigned char *)ctx->adj_mem[k ? 12 : 7];
        A.sets[k] = {ctx->adj_mem[k ? 11 : 6], (double *)ctx->adj_mem[13 + k], fl, fl + (size_t)nb * kBS3};
    }
    double *xpart = (double *)ctx->adj_mem[9];
    A.slots.assign(p->nsnapshots, nullptr);
    for (int i = 0; i < p->nsnapshots; i++) A.slots[i] = (Real *)((char *)ctx->adj_mem[10] + A.fbytes * (size_t)i);
    e = cudaMemsetAsync(A.grad_acc, 0, (size_t)nb * kGradSlots * sizeof(double), ctx->stream);
    // forward steps on the pipelined kernel where it applies (bit-identical)
    A.X0 = X0;
    A.abs_terms = (p->flags & GBFK_ADJ_TERM_MAGNITUDES) != 0;
    if (e == cudaSuccess && tma_step_eligible<Real>(A.v) && ctx->step_pref != GBFK_STEP_BLOCK) {
        rc = build_step_lists(ctx);
        if (rc) {
            cleanup();
            return rc;
        }
        A.lists = {ctx->d_lists, ctx->n_heavy, ctx->d_lists + ctx->n_heavy, ctx->n_empty};
        // which blocks are empty changes with the lists: buffers known to hold
        // +0 in the old empty blocks are not known to in the new ones
        if (ctx->adj_clean_gen != ctx->lists_gen) {
            ctx->adj_clean.clear();
            ctx->adj_clean_gen = ctx->lists_gen;
        }
        if (fresh) {
            ctx->adj_clean.insert({(const void *)F, (const void *)A.T0, (const void *)A.T1, (const void *)A.T2});
            for (Real *b : A.slots) ctx->adj_clean.insert(b);
        }
        const double h = sizeof(Real) == 8 ? ctx->h_h[0] : (double)(float)ctx->h_h[0];
        A.ih2 = 1. / (h * h);
        const Real *inputs[] = {X0, A.T0, A.T1};
        for (const Real *b : inputs)
            if (e == cudaSuccess) e = A.add_maps(b);
        for (Real *b : A.slots)
            if (e == cudaSuccess) e = A.add_maps(b);
        A.pipelined = e == cudaSuccess;
    }
    // initial condition
    if (e == cudaSuccess) {
        if (p->sigma > 0) {
            e = launch_gaussian_ic<Real>(bpd, (const Real *)ctx->pw, (const Real *)ctx->pg, p->x0, p->sigma, X0,
                                         ctx->stream);
            ctx->launches++;
        } else {
            e = cudaMemcpyAsync(X0, ctx->phi[ctx->cur], A.fbytes, cudaMemcpyDeviceToDevice, ctx->stream);
        }
    }
    // the blocks the adjoint steps run: a block can hold a domain cell only if
    // it has tissue (a heavy block) or a positive initial value (a kEmpty cell
    // at +0 stays +0 and outside the domain).  The others have lambda = mu = 0
    // at every step: their cells are outside the domain with phi = +0, so
    // mu = lambda' [0 < phi <= 1] = 0, and every face coefficient that
    // couples them to a neighbour is exactly 0 (a kBlockEmpty block's cells
    // and face halos have p_w = p_g = 0, so both diffusivities of such a face
    // are 0 and its harmonic mean is 0), so no neighbour feeds their lambda.
    // They keep status kAdjMuZero in both sets and lambda 0.
    bool ic_clean = false;  // every empty block of the initial condition holds +0
    if (e == cudaSuccess && ctx->identity_slots) {
        int *d_list = (int *)ctx->adj_mem[15];
        unsigned char *d_pos = (unsigned char *)(d_list + nb);
        std::vector<unsigned char> bt(nb), pos(nb);
        e = launch_block_any_positive<Real>(X0, nb, d_pos, ctx->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(pos.data(), d_pos, nb, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(bt.data(), ctx->d_btype, nb, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        ctx->launches++;
        if (e == cudaSuccess) {
            ic_clean = true;
            for (int b = 0; b < nb; b++)
                if (bt[b] == kBlockEmpty && pos[b]) ic_clean = false;
            // blocks with tissue first, then empty blocks with a positive
            // initial value (a tumour outside the anatomy)
            std::vector<int> list;
            for (int b = 0; b < nb; b++)
                if (bt[b] != kBlockEmpty) list.push_back(b);
            for (int b = 0; b < nb; b++)
                if (bt[b] == kBlockEmpty && pos[b]) list.push_back(b);
            if (!list.empty() && (int)list.size() < nb) {
                e = cudaMemcpyAsync(d_list, list.data(), list.size() * sizeof(int), cudaMemcpyHostToDevice,
                                    ctx->stream);
                for (int k = 0; k < 2 && e == cudaSuccess; k++)
                    e = cudaMemsetAsync(A.sets[k].status, kAdjMuZero, nb, ctx->stream);
                A.blocks = d_list;
                A.nlaunch = (int)list.size();
            }
        }
    }
    // forward steps skip the empty blocks where that gives the same bits; a
    // tumour outside the anatomy (or a non-finite dt) may write into them,
    // after which no buffer is known to hold +0 there
    A.skip_empty = e == cudaSuccess && A.pipelined && ic_clean && std::isfinite(p->dt);
    if (!A.skip_empty) ctx->adj_clean.clear();  // full steps: nothing is tracked
    // forward to the horizon (storing the first chain of checkpoints), loss and its gradient
    if (e == cudaSuccess) {
        A.join(ctx->stream, A.fs);
        A.sweep(X0, F, p->nsteps, p->nsnapshots);
        A.adjoint_reads(F);
        e = A.err;
    }
    double lik[4] = {0, 0, 0, 0};
    if (e == cudaSuccess) {
        if (!ctx->d_partial) e = cudaMalloc(&ctx->d_partial, (size_t)148 * 4 * 7 * sizeof(double));
        if (e == cudaSuccess && !ctx->d_lik) e = cudaMalloc(&ctx->d_lik, 4 * sizeof(double));
        if (e == cudaSuccess && ctx->model_bytes < (size_t)n * n * n * sizeof(double)) {
            if (ctx->d_model) cudaFree(ctx->d_model);
            ctx->d_model = nullptr;
            ctx->model_bytes = 0;
            e = cudaMalloc(&ctx->d_model, (size_t)n * n * n * sizeof(double));
            if (e == cudaSuccess) ctx->model_bytes = (size_t)n * n * n * sizeof(double);
        }
    }
    if (e == cudaSuccess)
        e = launch_uq_dump<Real>(ctx->d_slot, (const Real *)ctx->d_origin, (const Real *)ctx->d_h, nb, F, n,
                                 ctx->d_model, ctx->stream);
    if (e == cudaSuccess) {
        LikelihoodParams lp;
        lp.pet_sigma2 = 1;
        lp.pet_scale = 1;
        lp.t1_uc = p->t1_uc;
        lp.t2_uc = p->t2_uc;
        lp.slope = p->slope;
        lp.step_pet = 1;
        lp.step_mri = 1;
        // with a ROI (HGG_Likelihood.cpp:97-124) the loss sums over its voxels only
        e = launch_likelihood(ctx->d_model, n, ctx->d_t1c, ctx->d_flair, nullptr, ctx->nroi ? ctx->d_roi : nullptr,
                              ctx->nroi, lp, ctx->d_partial, 148 * 4, ctx->d_lik, ctx->stream);
        ctx->launches += 3;
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(lik, ctx->d_lik, 4 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
    int *roi_count = nullptr;
    if (e == cudaSuccess && ctx->nroi) {
        if (ctx->roi_count_bytes < (size_t)n * n * n * sizeof(int)) {
            if (ctx->d_roi_count) cudaFree(ctx->d_roi_count);
            ctx->d_roi_count = nullptr;
            ctx->roi_count_bytes = 0;
            e = cudaMalloc(&ctx->d_roi_count, (size_t)n * n * n * sizeof(int));
            if (e == cudaSuccess) ctx->roi_count_bytes = (size_t)n * n * n * sizeof(int);
        }
        if (e == cudaSuccess) e = launch_roi_count(n, ctx->d_roi, ctx->nroi, ctx->d_roi_count, ctx->stream);
        roi_count = ctx->d_roi_count;
        ctx->launches++;
    }
    if (e == cudaSuccess) {
        e = launch_loss_grad<Real>(bpd, F, ctx->d_t1c, ctx->d_flair, roi_count, p->t1_uc, p->t2_uc, p->slope, A.LAM,
                                   ctx->stream);
        ctx->launches++;
    }
    // reverse sweep, then lambda_0 into LAM
    if (e == cudaSuccess) {
        A.reverse_chain(0, p->nsteps, p->nsnapshots, X0);
        e = A.err;
    }
    if (e == cudaSuccess) {
        A.finish();
        A.join(A.fs, ctx->stream);
        e = A.err;
    }
    // parameter gradients
    std::vector<double> acc((size_t)nb * kGradSlots);
    std::vector<double> xp((size_t)xparts * 6, 0.0);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(acc.data(), A.grad_acc, acc.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess && p->sigma > 0) {
        e = launch_x0_grad<Real>(bpd, X0, A.LAM, p->x0, p->sigma, xpart, xparts, ctx->stream);
        ctx->launches++;
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(xp.data(), xpart, xp.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
    }
    if (e == cudaSuccess && grad_c0) {
        if (ctx->stage_bytes < A.fbytes) {
            if (ctx->d_stage) cudaFree(ctx->d_stage);
            ctx->d_stage = nullptr;
            ctx->stage_bytes = 0;
            e = cudaMalloc(&ctx->d_stage, A.fbytes);
            if (e == cudaSuccess) ctx->stage_bytes = A.fbytes;
        }
        if (e == cudaSuccess) e = launch_dense_scatter<Real>(A.LAM, (Real *)ctx->d_stage, n, false, ctx->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(grad_c0, ctx->d_stage, A.fbytes, cudaMemcpyDeviceToHost, ctx->stream);
        ctx->launches++;
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cleanup();
    if (e != cudaSuccess) return fail(ctx, GBFK_E_CUDA, "forward_adjoint: %s", cudaGetErrorString(e));
    auto nsum = [](const double *v, size_t stride, size_t count) {
        double s = 0, c = 0;
        for (size_t i = 0; i < count; i++)
            for (int k = 0; k < 2; k++) {
                const double x = v[i * stride + k];
                const double t = s + x;
                if (fabs(s) >= fabs(x)) c += (s - t) + x;
                else c += (x - t) + s;
                s = t;
            }
        return s + c;
    };
    res->loss = -(lik[1] + lik[2]);
    res->drho = nsum(acc.data(), kGradSlots, nb);
    res->dDw = nsum(acc.data() + 2, kGradSlots, nb);
    res->drho_abs = res->dDw_abs = 0;
    if (A.abs_terms)
        for (int b = 0; b < nb; b++) {
            res->drho_abs += acc[(size_t)b * kGradSlots + 4];
            res->dDw_abs += acc[(size_t)b * kGradSlots + 5];
        }
    for (int d = 0; d < 3; d++) res->dx0[d] = p->sigma > 0 ? nsum(xp.data() + 2 * d, 6, xparts) : 0.0;
    res->forward_steps = A.fsteps;
    res->adjoint_steps = A.asteps;
    return GBFK_OK;
}

}  // namespace

extern "C" int gbfk_forward_adjoint(gbfk_ctx *ctx, const gbfk_adjoint_params *p, gbfk_adjoint_result *out,
                                    void *grad_c0)
{
    if (!ctx) return GBFK_E_INVALID;
    ctx->phi_clamped = false;
    if (!p || !out) return fail(ctx, GBFK_E_INVALID, "forward_adjoint: null argument");
    if (!ctx->uniform || !ctx->have_origin) return fail(ctx, GBFK_E_STATE, "forward_adjoint: needs a uniform power-of-two grid");
    if (ctx->obs_n != 8 * ctx->bpd) return fail(ctx, GBFK_E_STATE, "forward_adjoint: observations must be on the grid");
    if (p->nsteps < 0 || p->nsnapshots < 1 || !(p->slope != 0) || !(p->Dw > 0) ||
        (p->flags & ~GBFK_ADJ_TERM_MAGNITUDES) != 0)
        return fail(ctx, GBFK_E_INVALID, "forward_adjoint: bad parameters");
    CK(cudaSetDevice(ctx->device));
    return ctx->precision == GBFK_F64 ? forward_adjoint_impl<double>(ctx, p, out, grad_c0)
                                      : forward_adjoint_impl<float>(ctx, p, out, grad_c0);
}
