// Batched TMCMC-stage forward solves.
//
// The reference evaluates a TMCMC stage as independent tasks
// (tools/pi4u_lite/Inference/engine_tmcmc.c:597-624), each forking a process
// that runs the whole solver on one parameter sample
// (tools/pi4u_lite/Inference/fitfun_glioma.c:46-245, runAll.sh: brain -UQ 1).
// Here all samples of a stage live in GPU memory and advance together: one
// launch per time step covers every sample that has not reached its own
// horizon.  Samples are sorted by step count (longest first), so the active
// samples of step k are a prefix and retired samples cost nothing.  Fields
// are stored by that sorted position: position p's pool is blocks
// p*nblocks .. (p+1)*nblocks-1 of one phi buffer per step parity and of one
// face-coefficient buffer, so one tensor map per parity covers the halos of
// every sample (the pipelined step, gbfk_step_tma.cu).
#include "gbfk.h"
#include "gbfk_exact.cuh"
#include "gbfk_host.h"
#include "gbfk_kernels.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <numeric>
#include <string>
#include <vector>

using namespace gbfk;

namespace gbfk {
cudaError_t upload_ghost_table();
}

struct gbfk_batch {
    int precision = GBFK_F32;
    size_t rsize = 4;
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int bpd = 0, n = 0, nblocks = 0;
    int max_samples = 0, max_anatomies = 0;
    int log2_bpd = -1;
    int *d_nbr = nullptr;
    double *d_ih2 = nullptr;
    // per anatomy (consecutive pools of pw_all, pg_all, meta_all, btype_all)
    void *pw_all = nullptr, *pg_all = nullptr;
    unsigned short *meta_all = nullptr;
    unsigned char *btype_all = nullptr;
    std::vector<void *> pw, pg;
    std::vector<unsigned short *> meta;
    std::vector<unsigned char *> btype;
    std::vector<bool> anatomy_set;
    // per sample (in the caller's order)
    int nsamples = 0;
    std::vector<gbfk_sample> params;
    // per position (sorted by horizon, longest first)
    void *phi_all[2] = {nullptr, nullptr};
    void *H_all = nullptr;
    std::vector<int> order;  // position -> caller's sample index
    std::vector<int> pos;    // caller's sample index -> position
    void *d_views = nullptr;
    unsigned *d_nan = nullptr;   // per position
    unsigned *d_err = nullptr;   // the pipelined step's error word
    // pipelined step: work lists, per-position parameters, tensor maps
    int *d_lists = nullptr;      // lists, list_off, hpref, epref, anatomy (one allocation)
    size_t lists_cap = 0;
    int2 *d_dec = nullptr;       // decoded heavy items, then decoded empty items
    size_t dec_cap = 0;
    BatchLists bl{};
    std::vector<int> h_hpref;    // host copy of bl.hpref
    // every sample's empty blocks hold +0 in both state buffers after the
    // first step and keep it (see batch_prepare); later steps skip them
    bool empties_static = false;
    void *d_rho = nullptr;
    double *d_dt = nullptr;
    double ih2 = 0;
    CUtensorMap maps[2][3];
    bool maps_ready = false;
    int chosen_spc = 0;          // block kernel: samples per CTA; -1: the pipelined kernel
    int chosen_shape = -1;       // pipelined kernel: launch shape code (-1: the default)
    int graph_launches = 0;      // CUDA graphs the last run replayed
    bool ran = false;            // the samples hold their final states
    // observations of the likelihood step (n^3 grid) and its scratch
    unsigned char *d_t1c = nullptr, *d_flair = nullptr;
    double *d_pet = nullptr;
    int *d_roi = nullptr;
    int nroi = 0;
    bool have_obs = false;
    double *d_model = nullptr;   // one sample's dump grid
    double *d_partial = nullptr; // likelihood partial sums
    double *d_lik = nullptr;     // 4 per sample
    // GBFK_IC_BALL samples: band cells (int64 pool index) and their values
    void *d_ball = nullptr;
    size_t ball_cap = 0;
    int64_t launches = 0;
    std::string err;
};

namespace {

int bfail(gbfk_batch *b, int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (b) b->err = buf;
    return code;
}

#define BK(call)                                                                                          \
    do {                                                                                                  \
        cudaError_t e_ = (call);                                                                          \
        if (e_ != cudaSuccess)                                                                            \
            return bfail(b, e_ == cudaErrorMemoryAllocation ? GBFK_E_OOM : GBFK_E_CUDA, "%s: %s (%s:%d)", \
                         #call, cudaGetErrorString(e_), __FILE__, __LINE__);                              \
    } while (0)

// One sample's phi (block-pool order of a uniform bpd^3 grid) as doubles on
// the n^3 grid, x fastest: the dump of a uniform grid at its own resolution
// (each cell written once, Glioma_ReactionDiffusion.cpp:208-262).
template <typename Real>
__global__ void pool_to_dense_kernel(const Real *__restrict__ pool, int n, double *__restrict__ out)
{
    const int64_t N = (int64_t)n * n * n;
    const int bpd = n / kBS;
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < N; g += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(g % n), y = (int)((g / n) % n), z = (int)(g / ((int64_t)n * n));
        const int64_t slot = (x >> 3) + (int64_t)bpd * ((y >> 3) + (int64_t)bpd * (z >> 3));
        out[g] = (double)pool[slot * kBS3 + (x & 7) + kBS * ((y & 7) + kBS * (z & 7))];
    }
}

template <typename Real>
PoolView<Real> batch_pool(gbfk_batch *b)
{
    PoolView<Real> v;
    v.slot = nullptr;
    v.nbr = b->d_nbr;
    v.hblk = nullptr;
    v.gpw = v.gpg = v.gphi = nullptr;
    v.pw = v.pg = nullptr;
    v.btype = nullptr;
    v.nblocks = b->nblocks;
    v.identity_slots = 1;
    v.log2_bpd = b->log2_bpd;
    return v;
}

// Tumour initial condition of a sample on the device: c0 = exp(-|x-x0|^2 /
// (2 sigma^2)) where p_w + p_g > 0, else 0, in Real, at vertex positions
// x = i / n (MRAG BlockInfo::pos); block-pool order.
template <typename Real>
__global__ void ic_kernel(int n, int bpd, const Real *__restrict__ pw, const Real *__restrict__ pg, double x0,
                          double y0, double z0, double sigma, Real *__restrict__ out)
{
    const int64_t N = (int64_t)n * n * n;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = i >> 9;
        const int c = (int)(i & 511);
        const int bx = (int)(b % bpd), by = (int)((b / bpd) % bpd), bz = (int)(b / ((int64_t)bpd * bpd));
        const double x = (double)(bx * 8 + (c & 7)) / n, y = (double)(by * 8 + ((c >> 3) & 7)) / n,
                     z = (double)(bz * 8 + (c >> 6)) / n;
        const double r2 = (x - x0) * (x - x0) + (y - y0) * (y - y0) + (z - z0) * (z - z0);
        const double v = exp(-r2 / (2. * sigma * sigma));
        out[i] = (pw[i] + pg[i] > (Real)0) ? (Real)v : (Real)0;
    }
}

// The reference's smoothed-ball tumour of a sample: the band cells computed
// on the host, scattered into the zeroed state where the cell has tissue.
template <typename Real>
__global__ void ball_ic_kernel(int count, const int64_t *__restrict__ cell, const Real *__restrict__ value,
                               const Real *__restrict__ pw, const Real *__restrict__ pg, Real *__restrict__ out)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const int64_t c = cell[i];
        out[c] = (pw[c] + pg[c] > (Real)0) ? value[i] : (Real)0;
    }
}

// Work lists of the pipelined step: per anatomy in use, its heavy blocks
// (block * 4 + type, mixed first) and empty blocks from the block types the
// face kernel wrote; per position its anatomy and the prefix sums of the
// list lengths.  Call after the face kernels of batch_prepare.
int batch_lists(gbfk_batch *b)
{
    const int nb = b->nblocks, na = b->max_anatomies, ns = b->nsamples;
    std::vector<int> used(na, 0);
    for (int k = 0; k < ns; k++) used[b->params[b->order[k]].anatomy] = 1;
    std::vector<int> lists, off(2 * na, 0), nh(na, 0), ne(na, 0);
    std::vector<unsigned char> bt(nb);
    for (int a = 0; a < na; a++) {
        if (!used[a]) continue;
        BK(cudaMemcpyAsync(bt.data(), b->btype[a], nb, cudaMemcpyDeviceToHost, b->stream));
        BK(cudaStreamSynchronize(b->stream));
        off[2 * a] = (int)lists.size();
        for (int q = 0; q < nb; q++)
            if (bt[q] == kBlockMixed) lists.push_back(q * 4 + kBlockMixed);
        for (int q = 0; q < nb; q++)
            if (bt[q] == kBlockTissue) lists.push_back(q * 4 + kBlockTissue);
        nh[a] = (int)lists.size() - off[2 * a];
        off[2 * a + 1] = (int)lists.size();
        for (int q = 0; q < nb; q++)
            if (bt[q] == kBlockEmpty) lists.push_back(q);
        ne[a] = (int)lists.size() - off[2 * a + 1];
        if (nh[a] + ne[a] != nb) return bfail(b, GBFK_E_CUDA, "batch: unknown block type");
    }
    std::vector<int> hpref(ns + 1, 0), epref(ns + 1, 0), anat(ns);
    for (int k = 0; k < ns; k++) {
        anat[k] = b->params[b->order[k]].anatomy;
        hpref[k + 1] = hpref[k] + nh[anat[k]];
        epref[k + 1] = epref[k] + ne[anat[k]];
    }
    // one allocation: lists | list_off | hpref | epref | anatomy
    const size_t need = lists.size() + off.size() + 2 * (size_t)(ns + 1) + ns;
    if (b->lists_cap < need) {
        if (b->d_lists) cudaFree(b->d_lists);
        b->d_lists = nullptr;
        b->lists_cap = 0;
        BK(cudaMalloc(&b->d_lists, need * sizeof(int)));
        b->lists_cap = need;
    }
    std::vector<int> all;
    all.reserve(need);
    all.insert(all.end(), lists.begin(), lists.end());
    all.insert(all.end(), off.begin(), off.end());
    all.insert(all.end(), hpref.begin(), hpref.end());
    all.insert(all.end(), epref.begin(), epref.end());
    all.insert(all.end(), anat.begin(), anat.end());
    BK(cudaMemcpyAsync(b->d_lists, all.data(), all.size() * sizeof(int), cudaMemcpyHostToDevice, b->stream));
    BK(cudaStreamSynchronize(b->stream));
    int *d = b->d_lists;
    b->bl.lists = d;
    b->bl.list_off = d + lists.size();
    b->bl.hpref = b->bl.list_off + off.size();
    b->bl.epref = b->bl.hpref + ns + 1;
    b->bl.anatomy = b->bl.epref + ns + 1;
    // every item decoded once: (position, entry) in global item order
    const size_t nitems = (size_t)hpref[ns] + (size_t)epref[ns];
    if (b->dec_cap < nitems) {
        if (b->d_dec) cudaFree(b->d_dec);
        b->d_dec = nullptr;
        b->dec_cap = 0;
        BK(cudaMalloc(&b->d_dec, std::max<size_t>(nitems, 1) * sizeof(int2)));
        b->dec_cap = nitems;
    }
    std::vector<int2> dec(nitems);
    for (int k = 0; k < ns; k++) {
        const int a = anat[k];
        for (int i = 0; i < nh[a]; i++) dec[(size_t)hpref[k] + i] = make_int2(k, lists[off[2 * a] + i]);
        for (int i = 0; i < ne[a]; i++)
            dec[(size_t)hpref[ns] + epref[k] + i] = make_int2(k, lists[off[2 * a + 1] + i] * 4);
    }
    if (nitems)
        BK(cudaMemcpyAsync(b->d_dec, dec.data(), nitems * sizeof(int2), cudaMemcpyHostToDevice, b->stream));
    BK(cudaStreamSynchronize(b->stream));
    b->bl.hdec = b->d_dec;
    b->bl.edec = b->d_dec + hpref[ns];
    b->h_hpref.swap(hpref);
    return GBFK_OK;
}

template <typename Real>
Real *pos_field(gbfk_batch *b, void *base, int p, int per_block)
{
    return (Real *)base + (int64_t)p * b->nblocks * per_block;
}

template <typename Real>
int batch_prepare(gbfk_batch *b)
{
    // positions: sorted by horizon, longest first
    b->order.resize(b->nsamples);
    std::iota(b->order.begin(), b->order.end(), 0);
    std::stable_sort(b->order.begin(), b->order.end(),
                     [&](int i, int j) { return b->params[i].nsteps > b->params[j].nsteps; });
    b->pos.assign(b->nsamples, 0);
    for (int k = 0; k < b->nsamples; k++) b->pos[b->order[k]] = k;
    // band cells of every GBFK_IC_BALL sample in pool order, one upload
    std::vector<int64_t> bcell;
    std::vector<Real> bval;
    std::vector<size_t> boff(b->nsamples + 1, 0);
    {
        std::vector<gbfk_host::BallCell<Real>> cells;
        const int bpd = b->bpd;
        for (int k = 0; k < b->nsamples; k++) {
            const gbfk_sample &p = b->params[b->order[k]];
            if (p.ic == GBFK_IC_BALL) {
                if (!gbfk_host::ball_band_cells<Real>(bpd, p.x0, cells))
                    return bfail(b, GBFK_E_INVALID, "sample %d: a cell in the ball's core", b->order[k]);
                for (const auto &c : cells) {
                    const int64_t slot = (c.x >> 3) + (int64_t)bpd * ((c.y >> 3) + (int64_t)bpd * (c.z >> 3));
                    bcell.push_back(slot * kBS3 + (c.x & 7) + 8 * ((c.y & 7) + 8 * (c.z & 7)));
                    bval.push_back(c.value);
                }
            }
            boff[k + 1] = bcell.size();
        }
    }
    const size_t nball = bcell.size();
    const size_t val_off = (nball * sizeof(int64_t) + 255) & ~(size_t)255;
    if (nball) {
        const size_t need = val_off + nball * sizeof(Real);
        if (need > b->ball_cap) {
            if (b->d_ball) BK(cudaFree(b->d_ball));
            b->d_ball = nullptr;
            b->ball_cap = 0;
            if (cudaMalloc(&b->d_ball, need) != cudaSuccess) {
                cudaGetLastError();
                return bfail(b, GBFK_E_OOM, "ball initial conditions: %zu bytes", need);
            }
            b->ball_cap = need;
        }
        BK(cudaMemcpyAsync(b->d_ball, bcell.data(), nball * sizeof(int64_t), cudaMemcpyHostToDevice, b->stream));
        BK(cudaMemcpyAsync((char *)b->d_ball + val_off, bval.data(), nball * sizeof(Real), cudaMemcpyHostToDevice,
                           b->stream));
    }
    // face coefficients and meta words of every sample's (anatomy, Dw, Dg);
    // initial conditions in the parity-0 buffer
    for (int k = 0; k < b->nsamples; k++) {
        const gbfk_sample &p = b->params[b->order[k]];
        PoolView<Real> v = batch_pool<Real>(b);
        v.pw = (const Real *)b->pw[p.anatomy];
        v.pg = (const Real *)b->pg[p.anatomy];
        v.btype = b->btype[p.anatomy];
        BK(launch_faces<Real>(v, (Real)p.Dw, (Real)p.Dg, pos_field<Real>(b, b->H_all, k, kFacesPerBlock),
                              b->meta[p.anatomy], b->btype[p.anatomy], b->stream));
        int64_t nb = ((int64_t)b->nblocks * kBS3 + 255) / 256;
        if (nb > 148 * 32) nb = 148 * 32;
        Real *phi0 = pos_field<Real>(b, b->phi_all[0], k, kBS3);
        if (p.ic == GBFK_IC_BALL) {
            BK(cudaMemsetAsync(phi0, 0, (size_t)b->nblocks * kBS3 * sizeof(Real), b->stream));
            const int count = (int)(boff[k + 1] - boff[k]);
            if (count > 0) {
                ball_ic_kernel<Real><<<(count + 255) / 256, 256, 0, b->stream>>>(
                    count, (const int64_t *)b->d_ball + boff[k], (const Real *)((char *)b->d_ball + val_off) + boff[k],
                    v.pw, v.pg, phi0);
                BK(cudaGetLastError());
                b->launches++;
            }
        } else {
            ic_kernel<Real><<<(int)nb, 256, 0, b->stream>>>(b->n, b->bpd, v.pw, v.pg, p.x0[0], p.x0[1], p.x0[2],
                                                             p.sigma, phi0);
            BK(cudaGetLastError());
            b->launches++;
        }
        b->launches++;
    }
    std::vector<SampleView<Real>> views(b->nsamples);
    std::vector<Real> rho(b->nsamples);
    std::vector<double> dt(b->nsamples);
    for (int k = 0; k < b->nsamples; k++) {
        const gbfk_sample &p = b->params[b->order[k]];
        SampleView<Real> &sv = views[k];
        sv.pw = (const Real *)b->pw[p.anatomy];
        sv.pg = (const Real *)b->pg[p.anatomy];
        sv.btype = b->btype[p.anatomy];
        sv.meta = b->meta[p.anatomy];
        sv.H = pos_field<Real>(b, b->H_all, k, kFacesPerBlock);
        sv.phi0 = pos_field<Real>(b, b->phi_all[0], k, kBS3);
        sv.phi1 = pos_field<Real>(b, b->phi_all[1], k, kBS3);
        sv.rho = (Real)p.rho;
        sv.dt = p.dt;
        sv.nsteps = p.nsteps;
        rho[k] = (Real)p.rho;
        dt[k] = p.dt;
    }
    BK(cudaMemcpyAsync(b->d_views, views.data(), views.size() * sizeof(SampleView<Real>), cudaMemcpyHostToDevice,
                       b->stream));
    BK(cudaMemcpyAsync(b->d_rho, rho.data(), rho.size() * sizeof(Real), cudaMemcpyHostToDevice, b->stream));
    BK(cudaMemcpyAsync(b->d_dt, dt.data(), dt.size() * sizeof(double), cudaMemcpyHostToDevice, b->stream));
    BK(cudaMemsetAsync(b->d_nan, 0, b->max_samples * sizeof(unsigned), b->stream));
    BK(cudaMemsetAsync(b->d_err, 0, sizeof(unsigned), b->stream));
    BK(cudaStreamSynchronize(b->stream));
    // An empty block (no tissue in it or its face halos: p_w = p_g = 0) starts
    // at +0 -- both initial conditions write +0 wherever p_w + p_g is not
    // positive -- and, with a finite dt, a kEmpty cell at +0 is outside the
    // domain and stays +0 (the update clamps it).  The first step writes
    // those +0 into the other state buffer; from then on both buffers hold
    // the final bits of every empty block, and the pipelined step skips them.
    b->empties_static = true;
    for (int k = 0; k < b->nsamples; k++)
        if (!std::isfinite(b->params[b->order[k]].dt)) b->empties_static = false;
    return b->log2_bpd >= 0 ? batch_lists(b) : GBFK_OK;
}

// One step of the batch with the chosen kernel: the pipelined step
// (spc == -1) or the per-block kernel with spc samples per CTA.
template <typename Real>
cudaError_t batch_step(gbfk_batch *b, const BatchView<Real> &bv, int nactive, int step, int spc, int shape)
{
    if (spc > 0) return launch_rd_batch_step<Real>(bv, nactive, step, spc, b->stream);
    const int par = step & 1;
    const bool skip = b->empties_static && step > 0;
    const int items = skip ? b->h_hpref[nactive] : nactive * b->nblocks;
    return launch_rd_batch_step_tma<Real>(
        b->bl, nactive, items, skip, b->log2_bpd, b->nblocks, (const Real *)b->phi_all[par],
        (Real *)b->phi_all[par ^ 1], (const Real *)b->H_all, (const Real *)b->pw_all, (const Real *)b->pg_all,
        b->meta_all, (const Real *)b->d_rho, b->d_dt, b->ih2, step > 0, b->d_nan, b->d_err, b->maps[par], shape,
        b->stream);
}

template <typename Real>
int batch_run(gbfk_batch *b, int spc)
{
    int rc = batch_prepare<Real>(b);
    if (rc) return rc;
    if (spc == -1 && b->log2_bpd < 0)
        return bfail(b, GBFK_E_STATE, "batch_run: the pipelined step needs a power-of-two block count per direction");
    if (b->log2_bpd >= 0 && !b->maps_ready) {
        for (int q = 0; q < 2; q++)
            BK(make_pool_tensor_maps(b->phi_all[q], b->max_samples * b->nblocks, (int)sizeof(Real), b->maps[q]));
        b->maps_ready = true;
    }
    BatchView<Real> bv;
    bv.pool = batch_pool<Real>(b);
    bv.samples = (const SampleView<Real> *)b->d_views;
    bv.ih2 = b->d_ih2;
    bv.nan_flags = b->d_nan;
    const int maxsteps = b->nsamples ? b->params[b->order[0]].nsteps : 0;
    // active samples of step k: a prefix of the sorted list
    std::vector<int> sorted_steps(b->nsamples);
    for (int k = 0; k < b->nsamples; k++) sorted_steps[k] = b->params[b->order[k]].nsteps;
    int nactive = b->nsamples;
    auto active_at = [&](int step) {
        while (nactive > 0 && sorted_steps[nactive - 1] <= step) nactive--;
        return nactive;
    };
    int step = 0;
    // autotuner: the pipelined step (power-of-two grids) in each of its
    // launch shapes (consumer warps, heavy and empty ring slots) and the
    // per-block kernel with 1, 2 or 4 samples per CTA, each timed on 3 real
    // steps after 1 warm-up (every choice gives the same bits), the fastest
    // kept
    int shape = -1;
    if (spc == 0) {
        std::vector<std::pair<int, int>> cands;  // (samples per CTA, shape)
        if (b->log2_bpd >= 0) {
            int codes[16];
            const int nc = tma_batch_shapes(codes, 16);
            cands.push_back({-1, -1});
            for (int i = 0; i < nc; i++) cands.push_back({-1, codes[i]});
        }
        cands.push_back({1, -1});
        cands.push_back({2, -1});
        cands.push_back({4, -1});
        float best = 1e30f;
        std::pair<int, int> best_c = cands[0];
        cudaEvent_t e0, e1;
        BK(cudaEventCreate(&e0));
        BK(cudaEventCreate(&e1));
        for (size_t ci = 0; ci < cands.size() && step + 4 <= maxsteps; ci++) {
            const int cs = cands[ci].first, csh = cands[ci].second;
            BK(batch_step<Real>(b, bv, active_at(step), step, cs, csh));
            step++;
            BK(cudaEventRecord(e0, b->stream));
            for (int r = 0; r < 3; r++, step++) BK(batch_step<Real>(b, bv, active_at(step), step, cs, csh));
            BK(cudaEventRecord(e1, b->stream));
            BK(cudaEventSynchronize(e1));
            float ms = 0;
            BK(cudaEventElapsedTime(&ms, e0, e1));
            b->launches += 4;
            if (ms < best) {
                best = ms;
                best_c = cands[ci];
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        spc = best_c.first;
        shape = best_c.second;
    }
    b->chosen_spc = spc;
    b->chosen_shape = spc == -1 ? shape : 0;
    b->ran = false;
    // the remaining steps: the first one directly, the rest captured as CUDA
    // graphs of up to kGraphSteps launches each and replayed on the batch's
    // stream (a stream that cannot be captured, such as the legacy default
    // stream, runs them directly)
    if (step < maxsteps) {
        BK(batch_step<Real>(b, bv, active_at(step), step, spc, shape));
        b->launches++;
        step++;
    }
    constexpr int kGraphSteps = 512;
    std::vector<cudaGraphExec_t> execs;
    bool graphs = true;
    while (step < maxsteps) {
        const int end = std::min(maxsteps, step + kGraphSteps);
        cudaGraph_t g = nullptr;
        cudaGraphExec_t ge = nullptr;
        if (graphs && cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            cudaGetLastError();
            graphs = false;
        }
        cudaError_t le = cudaSuccess;
        for (int k = step; k < end && le == cudaSuccess; k++) le = batch_step<Real>(b, bv, active_at(k), k, spc, shape);
        if (graphs) {
            const cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
            if (le == cudaSuccess) le = ce;
            if (le == cudaSuccess) le = cudaGraphInstantiate(&ge, g, 0);
            if (g) cudaGraphDestroy(g);
            if (le == cudaSuccess) le = cudaGraphLaunch(ge, b->stream);
            if (ge) execs.push_back(ge);
        }
        if (le != cudaSuccess) {
            cudaStreamSynchronize(b->stream);
            for (cudaGraphExec_t x : execs) cudaGraphExecDestroy(x);
            return bfail(b, GBFK_E_CUDA, "batch_run: steps %d..%d: %s", step, end, cudaGetErrorString(le));
        }
        b->launches += end - step;
        step = end;
    }
    b->graph_launches = (int)execs.size();
    const cudaError_t se = cudaStreamSynchronize(b->stream);
    for (cudaGraphExec_t x : execs) cudaGraphExecDestroy(x);
    BK(se);
    unsigned err = 0;
    BK(cudaMemcpy(&err, b->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (err) return bfail(b, GBFK_E_TIMEOUT, "batch_run: a wait of the pipelined step timed out (1 s)");
    b->ran = true;  // final states, NaN ones included
    std::vector<unsigned> flags(b->nsamples);
    BK(cudaMemcpy(flags.data(), b->d_nan, b->nsamples * sizeof(unsigned), cudaMemcpyDeviceToHost));
    for (int k = 0; k < b->nsamples; k++)
        if (flags[k]) return bfail(b, GBFK_E_NAN, "sample %d became NaN", b->order[k]);
    return GBFK_OK;
}

template <typename Real>
int batch_likelihood(gbfk_batch *b, const gbfk_likelihood_params *params, int per_sample, double *out)
{
    const int n = b->n, nparts = 148 * 4;
    const size_t N = (size_t)n * n * n;
    if (!b->d_model) BK(cudaMalloc(&b->d_model, N * sizeof(double)));
    if (!b->d_partial) BK(cudaMalloc(&b->d_partial, (size_t)nparts * 7 * sizeof(double)));
    if (!b->d_lik) BK(cudaMalloc(&b->d_lik, (size_t)b->max_samples * 4 * sizeof(double)));
    const size_t field = (size_t)b->nblocks * kBS3;
    int64_t grid = (N + 255) / 256;
    if (grid > 148 * 32) grid = 148 * 32;
    for (int s = 0; s < b->nsamples; s++) {
        const gbfk_likelihood_params *p = params + (per_sample ? s : 0);
        LikelihoodParams lp;
        lp.pet_sigma2 = p->pet_sigma2;
        lp.pet_scale = p->pet_scale;
        lp.t1_uc = p->t1_uc;
        lp.t2_uc = p->t2_uc;
        lp.slope = p->slope;
        lp.step_pet = p->step_pet;
        lp.step_mri = p->step_mri;
        const Real *final = (const Real *)b->phi_all[b->params[s].nsteps & 1] + (size_t)b->pos[s] * field;
        pool_to_dense_kernel<Real><<<(int)grid, 256, 0, b->stream>>>(final, n, b->d_model);
        BK(cudaGetLastError());
        BK(launch_likelihood(b->d_model, n, b->d_t1c, b->d_flair, b->d_pet, b->nroi ? b->d_roi : nullptr, b->nroi,
                             lp, b->d_partial, nparts, b->d_lik + 4 * (size_t)s, b->stream));
        b->launches += 3;
    }
    BK(cudaMemcpyAsync(out, b->d_lik, (size_t)b->nsamples * 4 * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
    BK(cudaStreamSynchronize(b->stream));
    return GBFK_OK;
}

}  // namespace

extern "C" {

int gbfk_batch_create(const gbfk_config *cfg, int bpd, int max_samples, int max_anatomies, gbfk_batch **out)
{
    if (!cfg || !out || bpd <= 0 || max_samples <= 0 || max_anatomies <= 0) return GBFK_E_INVALID;
    if (cfg->precision != GBFK_F64 && cfg->precision != GBFK_F32) return GBFK_E_INVALID;
    *out = nullptr;
    gbfk_batch *b = new gbfk_batch();
    b->precision = cfg->precision;
    b->rsize = cfg->precision == GBFK_F64 ? 8 : 4;
    b->device = cfg->device;
    b->bpd = bpd;
    b->n = 8 * bpd;
    b->nblocks = bpd * bpd * bpd;
    b->max_samples = max_samples;
    b->max_anatomies = max_anatomies;
    auto bail = [&](int rc) {
        gbfk_batch_destroy(b);
        return rc;
    };
    if (cudaSetDevice(cfg->device) != cudaSuccess) return bail(GBFK_E_CUDA);
    if (upload_ghost_table() != cudaSuccess) return bail(GBFK_E_CUDA);
    if (cfg->stream) b->stream = (cudaStream_t)cfg->stream;
    else {
        if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(GBFK_E_CUDA);
        b->own_stream = true;
    }
    if ((bpd & (bpd - 1)) == 0) {
        int L = 0;
        while ((1 << L) < bpd) L++;
        b->log2_bpd = L;
    }
    const int nb = b->nblocks;
    std::vector<int> nbr((size_t)nb * 6);
    for (int bz = 0; bz < bpd; bz++)
        for (int by = 0; by < bpd; by++)
            for (int bx = 0; bx < bpd; bx++) {
                auto id = [&](int x, int y, int z) {
                    x = (x + bpd) % bpd; y = (y + bpd) % bpd; z = (z + bpd) % bpd;
                    return x + bpd * (y + bpd * z);
                };
                int *q = &nbr[(size_t)(bx + bpd * (by + bpd * bz)) * 6];
                q[0] = id(bx - 1, by, bz); q[1] = id(bx + 1, by, bz);
                q[2] = id(bx, by - 1, bz); q[3] = id(bx, by + 1, bz);
                q[4] = id(bx, by, bz - 1); q[5] = id(bx, by, bz + 1);
            }
    const double h = b->precision == GBFK_F64 ? 1.0 / (8.0 * bpd) : (double)(float)(1.0 / (8.0 * bpd));
    b->ih2 = 1. / (h * h);
    std::vector<double> ih2(nb, b->ih2);
    const size_t field = (size_t)nb * kBS3 * b->rsize;
    if (cudaMalloc(&b->d_nbr, nbr.size() * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&b->d_ih2, nb * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&b->d_views, (size_t)max_samples * sizeof(SampleView<double>)) != cudaSuccess ||
        cudaMalloc(&b->d_nan, (size_t)max_samples * sizeof(unsigned)) != cudaSuccess ||
        cudaMalloc(&b->d_err, sizeof(unsigned)) != cudaSuccess ||
        cudaMalloc(&b->d_rho, (size_t)max_samples * b->rsize) != cudaSuccess ||
        cudaMalloc((void **)&b->d_dt, (size_t)max_samples * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        return bail(GBFK_E_OOM);
    }
    cudaMemcpy(b->d_nbr, nbr.data(), nbr.size() * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(b->d_ih2, ih2.data(), nb * sizeof(double), cudaMemcpyHostToDevice);
    const size_t na = (size_t)max_anatomies, ns = (size_t)max_samples;
    if (cudaMalloc(&b->pw_all, na * field) != cudaSuccess || cudaMalloc(&b->pg_all, na * field) != cudaSuccess ||
        cudaMalloc(&b->meta_all, na * nb * kBS3 * sizeof(unsigned short)) != cudaSuccess ||
        cudaMalloc(&b->btype_all, na * nb) != cudaSuccess || cudaMalloc(&b->phi_all[0], ns * field) != cudaSuccess ||
        cudaMalloc(&b->phi_all[1], ns * field) != cudaSuccess ||
        cudaMalloc(&b->H_all, ns * nb * kFacesPerBlock * b->rsize) != cudaSuccess) {
        cudaGetLastError();
        return bail(GBFK_E_OOM);
    }
    b->pw.assign(max_anatomies, nullptr);
    b->pg.assign(max_anatomies, nullptr);
    b->meta.assign(max_anatomies, nullptr);
    b->btype.assign(max_anatomies, nullptr);
    b->anatomy_set.assign(max_anatomies, false);
    for (int a = 0; a < max_anatomies; a++) {
        b->pw[a] = (char *)b->pw_all + a * field;
        b->pg[a] = (char *)b->pg_all + a * field;
        b->meta[a] = b->meta_all + (size_t)a * nb * kBS3;
        b->btype[a] = b->btype_all + (size_t)a * nb;
    }
    *out = b;
    return GBFK_OK;
}

int gbfk_batch_destroy(gbfk_batch *b)
{
    if (!b) return GBFK_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    void *ptrs[] = {b->d_nbr,       b->d_ih2,    b->d_views, b->d_nan,      b->d_err,     b->d_rho, b->d_dt,
                    b->d_lists,     b->pw_all,   b->pg_all,  b->meta_all,   b->btype_all, b->phi_all[0],
                    b->phi_all[1],  b->H_all,    b->d_t1c,   b->d_flair,    b->d_pet,     b->d_roi, b->d_model,
                    b->d_partial,   b->d_lik,    b->d_ball,  b->d_dec};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return GBFK_OK;
}

const char *gbfk_batch_last_error(const gbfk_batch *b) { return b ? b->err.c_str() : "null batch"; }

int64_t gbfk_batch_launch_count(const gbfk_batch *b) { return b ? b->launches : 0; }

int gbfk_batch_set_anatomy(gbfk_batch *b, int anatomy, const void *pw_dense, const void *pg_dense)
{
    if (!b) return GBFK_E_INVALID;
    if (anatomy < 0 || anatomy >= b->max_anatomies || !pw_dense || !pg_dense)
        return bfail(b, GBFK_E_INVALID, "set_anatomy: bad anatomy index or null field");
    BK(cudaSetDevice(b->device));
    const size_t bytes = (size_t)b->n * b->n * b->n * b->rsize;
    void *stage = nullptr;
    BK(cudaMalloc(&stage, bytes));
    const void *src[2] = {pw_dense, pg_dense};
    void *dst[2] = {b->pw[anatomy], b->pg[anatomy]};
    for (int f = 0; f < 2; f++) {
        cudaError_t e = cudaMemcpyAsync(stage, src[f], bytes, cudaMemcpyHostToDevice, b->stream);
        if (e == cudaSuccess)
            e = b->precision == GBFK_F64
                    ? launch_dense_scatter<double>((const double *)stage, (double *)dst[f], b->n, true, b->stream)
                    : launch_dense_scatter<float>((const float *)stage, (float *)dst[f], b->n, true, b->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
        if (e != cudaSuccess) {
            cudaFree(stage);
            BK(e);
        }
        b->launches++;
    }
    cudaFree(stage);
    b->anatomy_set[anatomy] = true;
    return GBFK_OK;
}

int gbfk_batch_set_samples(gbfk_batch *b, int nsamples, const gbfk_sample *samples)
{
    if (!b) return GBFK_E_INVALID;
    if (nsamples < 0 || nsamples > b->max_samples || (nsamples && !samples))
        return bfail(b, GBFK_E_INVALID, "set_samples: %d samples for %d slots", nsamples, b->max_samples);
    for (int s = 0; s < nsamples; s++) {
        const gbfk_sample &p = samples[s];
        if (p.anatomy < 0 || p.anatomy >= b->max_anatomies || !b->anatomy_set[p.anatomy])
            return bfail(b, GBFK_E_STATE, "sample %d: anatomy %d not set", s, p.anatomy);
        if (p.ic != GBFK_IC_GAUSSIAN && p.ic != GBFK_IC_BALL)
            return bfail(b, GBFK_E_INVALID, "sample %d: initial condition %d", s, p.ic);
        if (p.nsteps < 0 || (p.ic == GBFK_IC_GAUSSIAN && !(p.sigma > 0)))
            return bfail(b, GBFK_E_INVALID, "sample %d: bad nsteps or sigma", s);
    }
    b->nsamples = nsamples;
    b->params.assign(samples, samples + nsamples);
    b->ran = false;
    return GBFK_OK;
}

int gbfk_batch_run(gbfk_batch *b, int samples_per_cta)
{
    if (!b) return GBFK_E_INVALID;
    if (samples_per_cta != -1 && samples_per_cta != 0 && samples_per_cta != 1 && samples_per_cta != 2 &&
        samples_per_cta != 4)
        return bfail(b, GBFK_E_INVALID, "samples_per_cta must be 0 (autotune), -1 (pipelined), 1, 2 or 4");
    BK(cudaSetDevice(b->device));
    return b->precision == GBFK_F64 ? batch_run<double>(b, samples_per_cta) : batch_run<float>(b, samples_per_cta);
}

int gbfk_batch_samples_per_cta(const gbfk_batch *b) { return b ? b->chosen_spc : 0; }

int gbfk_batch_tile_shape(const gbfk_batch *b, int shape[3])
{
    if (!b || !shape) return GBFK_E_INVALID;
    if (b->chosen_spc != -1) {
        shape[0] = shape[1] = shape[2] = 0;
        return GBFK_OK;
    }
    const int code = tma_shape_effective(b->chosen_shape, (int)b->rsize);
    shape[0] = code / 1000;
    shape[1] = (code / 100) % 10;
    shape[2] = code % 100;
    return GBFK_OK;
}

int gbfk_batch_graph_count(const gbfk_batch *b) { return b ? b->graph_launches : 0; }

int gbfk_batch_download(gbfk_batch *b, int sample, void *dense_out)
{
    if (!b) return GBFK_E_INVALID;
    if (sample < 0 || sample >= b->nsamples || !dense_out) return bfail(b, GBFK_E_INVALID, "download: bad sample");
    BK(cudaSetDevice(b->device));
    const size_t bytes = (size_t)b->n * b->n * b->n * b->rsize;
    void *stage = nullptr;
    BK(cudaMalloc(&stage, bytes));
    if (b->pos.size() != (size_t)b->nsamples) return bfail(b, GBFK_E_STATE, "download: the batch has not run");
    const size_t field = (size_t)b->nblocks * kBS3 * b->rsize;
    const void *src = (const char *)b->phi_all[b->params[sample].nsteps & 1] + (size_t)b->pos[sample] * field;
    cudaError_t e = b->precision == GBFK_F64
                        ? launch_dense_scatter<double>((const double *)src, (double *)stage, b->n, false, b->stream)
                        : launch_dense_scatter<float>((const float *)src, (float *)stage, b->n, false, b->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dense_out, stage, bytes, cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    cudaFree(stage);
    BK(e);
    b->launches++;
    return GBFK_OK;
}

int gbfk_batch_set_observations(gbfk_batch *b, const double *t1c, const double *flair, const double *pet,
                                const int *roi, int nroi)
{
    if (!b) return GBFK_E_INVALID;
    if (!t1c || !flair || nroi < 0 || (nroi > 0 && !roi))
        return bfail(b, GBFK_E_INVALID, "batch_set_observations: bad arguments");
    BK(cudaSetDevice(b->device));
    BK(cudaStreamSynchronize(b->stream));
    const int n = b->n;
    const size_t N = (size_t)n * n * n;
    for (int i = 0; i < 3 * nroi; i++)
        if (roi[i] < 0 || roi[i] >= n) return bfail(b, GBFK_E_INVALID, "batch_set_observations: ROI point out of the grid");
    void *old[] = {b->d_t1c, b->d_flair, b->d_pet, b->d_roi};
    for (void *q : old)
        if (q) cudaFree(q);
    b->d_t1c = b->d_flair = nullptr;
    b->d_pet = nullptr;
    b->d_roi = nullptr;
    b->have_obs = false;
    std::vector<unsigned char> a(N), c(N);
    for (size_t i = 0; i < N; i++) {
        a[i] = t1c[i] == 1 ? 1 : 0;  // HGG_Likelihood.cpp:141-148: a voxel counts where the mask equals 1
        c[i] = flair[i] == 1 ? 1 : 0;
    }
    BK(cudaMalloc(&b->d_t1c, N));
    BK(cudaMalloc(&b->d_flair, N));
    BK(cudaMemcpy(b->d_t1c, a.data(), N, cudaMemcpyHostToDevice));
    BK(cudaMemcpy(b->d_flair, c.data(), N, cudaMemcpyHostToDevice));
    if (pet) {
        BK(cudaMalloc(&b->d_pet, N * sizeof(double)));
        BK(cudaMemcpy(b->d_pet, pet, N * sizeof(double), cudaMemcpyHostToDevice));
    }
    if (roi && nroi > 0) {
        BK(cudaMalloc(&b->d_roi, (size_t)nroi * 3 * sizeof(int)));
        BK(cudaMemcpy(b->d_roi, roi, (size_t)nroi * 3 * sizeof(int), cudaMemcpyHostToDevice));
    }
    b->nroi = roi ? nroi : 0;
    b->have_obs = true;
    return GBFK_OK;
}

int gbfk_batch_log_likelihood(gbfk_batch *b, const gbfk_likelihood_params *params, int per_sample, double *out)
{
    if (!b) return GBFK_E_INVALID;
    if (!params || !out) return bfail(b, GBFK_E_INVALID, "batch_log_likelihood: null argument");
    if (!b->have_obs) return bfail(b, GBFK_E_STATE, "batch_log_likelihood: no observations");
    if (!b->ran) return bfail(b, GBFK_E_STATE, "batch_log_likelihood: the batch has not run");
    for (int s = 0; s < (per_sample ? b->nsamples : 1); s++) {
        const gbfk_likelihood_params *p = params + s;
        if (p->step_pet <= 0 || p->step_mri <= 0 || !(p->slope != 0))
            return bfail(b, GBFK_E_INVALID, "batch_log_likelihood: bad parameters (set %d)", s);
    }
    BK(cudaSetDevice(b->device));
    return b->precision == GBFK_F64 ? batch_likelihood<double>(b, params, per_sample, out)
                                    : batch_likelihood<float>(b, params, per_sample, out);
}

}  // extern "C"
