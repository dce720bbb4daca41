// The fused RD step as a persistent, TMA-fed pipeline, for uniform periodic
// power-of-two grids whose blocks sit in consecutive pool slots: one solve
// (gbfk_set_uniform; gbfk_rd_step) or every active sample of a TMCMC batch
// (gbfk_batch_run).  Results are bit-identical to rd_step_kernel and
// rd_batch_step_kernel (gbfk_kernels.cu), which step every other topology.
//
// Work items.  An item is one block of one sample.  Heavy items (mixed and
// tissue blocks: they need halos and face coefficients) and empty items
// (every cell and face-halo cell kEmpty: only the clamp of the update
// applies) are numbered globally by a work source (PoolSource: the host's
// block lists of one solve; BatchSource: per-anatomy block lists
// concatenated over the active samples).  CTA c of G (all resident) takes
// global items c, c + G, ... of each kind, so every CTA gets the same number
// of items of each kind, and runs its heavy and empty items merged evenly in
// time (order by (2j + 1) / n within each kind), so that the compute of
// heavy blocks overlaps the streaming of empty ones.
//
// Two rings of shared memory.  A heavy item lands in a heavy slot: its phi
// (cp.async.bulk), its six face halos as tensor boxes of the neighbouring
// blocks (cp.async.bulk.tensor.4d on the pool viewed as [slot][z][y][x],
// slot = sample * blocks + block; x faces as 4-wide boxes so that the inner
// extent is 16 bytes, y and z faces as a row set / a plane), its 1728 face
// coefficients and, for mixed blocks, its meta words.  An empty item's phi
// (2 KB in FP32) lands in an empty slot.  Warp kWarps is the producer: its
// 32 lanes decode the next 32 items of each kind in parallel, and lane 0
// issues every item in the merged order into its ring's next slot once that
// slot is released, with a (sample, block) header, completing on the slot's
// `full` mbarrier.
//
// Consumers.  All kWarps consumer warps compute a heavy item: consumer
// thread t owns the column x = t % 8, y = (t / 8) % 8 and kCells consecutive
// z from (t / 64) * kCells (a warp reads 32 consecutive cells of a z plane --
// no bank conflicts -- and stores 32 consecutive cells); the slot is free
// when all of them have released it.  Empty item j is computed by warp
// j % kWarps alone, in 16-byte vectors, and lives in empty slot
// j % kEmptySlots; kEmptySlots is a multiple of kWarps, so each empty slot
// serves one warp, which observes every phase of it in order (parity waits
// stay exact).  All waits are bounded: a wait that gives up sets the error
// word; the producer lets its copies in flight land (also bounded) before
// the CTA exits.  No load uses cluster multicast.
#include <cuda.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <vector>

#include "gbfk.h"
#include "gbfk_exact.cuh"
#include "gbfk_kernels.cuh"

namespace gbfk {
namespace {

constexpr unsigned long long kWaitNs = 1000000000ull;  // a stage not complete after 1 s is declared lost

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// One try_wait that may suspend the thread until the phase completes, for
// at most about kSuspendNs (a hint: the thread may wake earlier).
constexpr uint32_t kSuspendNs = 100000;

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(kSuspendNs)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// bounded wait for the phase of the given parity; true when it completed.
// The bound is kWaitNs of device time, and independently 2^24 polls.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity)
{
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    for (int i = 0; i < (1 << 24); i++) {
        if (mbar_try_wait(bar, parity)) return true;
        if (global_ns() - t0 > kWaitNs) return false;
    }
    return false;
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void box_g2s(void *dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                        uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
        : "memory");
}

// One slot of the heavy ring.  Every member starts on a 128-byte boundary
// (sizes are multiples of 128 bytes for float and double).
template <typename Real>
struct alignas(128) HeavySlot {
    Real in[512];           // the block, [z][y][x]
    Real xm[256], xp[256];  // x faces: [z][y][4] boxes of the x- (x = 4..7) / x+ (x = 0..3) neighbour
    Real ym[64], yp[64];    // y faces [z][x]: row y = 7 of the y- / y = 0 of the y+ neighbour
    Real zm[64], zp[64];    // z faces [y][x]: plane z = 7 of the z- / z = 0 of the z+ neighbour
    Real H[kFacesPerBlock];
    unsigned short meta[512];
};
static_assert(sizeof(HeavySlot<float>) % 128 == 0 && sizeof(HeavySlot<double>) % 128 == 0, "slot alignment");

// Items of one CTA that a one-pool launch stages in shared memory (a batch
// decodes its items 32 at a time instead).
constexpr int kMaxItems = 1024;

// What the producer tells the consumers about the item in a slot: its
// sample position, block * 4 + block type, and the sample's dt and rho.
struct alignas(16) SlotHdr {
    double dt, rho;
    int p, e;
};

// dynamic shared memory: heavy ring, empty ring, barriers, slot headers
template <typename Real, int kHeavySlots, int kEmptySlots>
struct SmemLayout {
    static constexpr size_t heavy = 0;
    static constexpr size_t empty = heavy + (size_t)kHeavySlots * sizeof(HeavySlot<Real>);
    static constexpr size_t bars = empty + (size_t)kEmptySlots * kBS3 * sizeof(Real);
    static constexpr size_t hdr = bars + (8 * (size_t)(2 * kHeavySlots + 2 * kEmptySlots + 2) + 127) / 128 * 128;
    static constexpr size_t items = hdr + sizeof(SlotHdr) * (size_t)(kHeavySlots + kEmptySlots);
    static constexpr size_t bytes = items + kMaxItems * sizeof(int);
};

// Merged item order of a CTA: true when item (jh, je) is the heavy one.
__device__ __forceinline__ bool heavy_next(int jh, int je, int nh, int ne)
{
    if (jh >= nh) return false;
    if (je >= ne) return true;
    return (int64_t)(2 * jh + 1) * ne <= (int64_t)(2 * je + 1) * nh;
}

// same-level periodic neighbour of block blk across face f on a 2^L grid
__device__ __forceinline__ int nb_of(int blk, int L, int f)
{
    const int m = (1 << L) - 1;
    int bx = blk & m, by = (blk >> L) & m, bz = blk >> (2 * L);
    const int d = f >> 1, s = (f & 1) ? 1 : -1;
    if (d == 0) bx = (bx + s) & m;
    else if (d == 1) by = (by + s) & m;
    else bz = (bz + s) & m;
    return bx | (by << L) | (bz << (2 * L));
}

// N consecutive Real from shared / to global memory in one 16- or 8-byte access
template <typename Real, int N>
__device__ __forceinline__ void vec_lds(const Real *src, Real (&d)[N])
{
    if constexpr (sizeof(Real) == 4 && N == 4) {
        const float4 a = *reinterpret_cast<const float4 *>(src);
        d[0] = a.x; d[1] = a.y; d[2] = a.z; d[3] = a.w;
    } else if constexpr (sizeof(Real) == 4 && N == 2) {
        const float2 a = *reinterpret_cast<const float2 *>(src);
        d[0] = a.x; d[1] = a.y;
    } else if constexpr (sizeof(Real) == 8 && N == 2) {
        const double2 a = *reinterpret_cast<const double2 *>(src);
        d[0] = a.x; d[1] = a.y;
    } else {
#pragma unroll
        for (int i = 0; i < N; i++) d[i] = src[i];
    }
}

template <typename Real, int N>
__device__ __forceinline__ void vec_stg(Real *dst, const Real (&d)[N])
{
    if constexpr (sizeof(Real) == 4 && N == 4) {
        *reinterpret_cast<float4 *>(dst) = make_float4(d[0], d[1], d[2], d[3]);
    } else if constexpr (sizeof(Real) == 4 && N == 2) {
        *reinterpret_cast<float2 *>(dst) = make_float2(d[0], d[1]);
    } else if constexpr (sizeof(Real) == 8 && N == 2) {
        *reinterpret_cast<double2 *>(dst) = make_double2(d[0], d[1]);
    } else {
#pragma unroll
        for (int i = 0; i < N; i++) dst[i] = d[i];
    }
}

// The face-box tensor maps (x, y, z faces) of one buffer of blocks, and the
// maps a launch reads: one set for one step; for a run of steps, the sets of
// the run's first input and of its two alternating buffers.
struct TmaMapSet {
    CUtensorMap m[3];
};
template <int N>
struct TmaMaps {
    TmaMapSet b[N];
};

// A run of steps in one launch (kMulti): step s reads in0 (s = 0) or
// buf[(s - 1) & 1] and writes buf[s & 1], except the last step, which writes
// last.  flags[c * kRunFlagStride]: the steps CTA c has stored (zero at
// launch); nbr[nbr_off[c] .. nbr_off[c + 1]): the other CTAs that own a face
// neighbour of one of CTA c's blocks.
template <typename Real>
struct StepRun {
    const Real *in0;
    Real *buf[2];
    Real *last;
    unsigned *flags;
    const int *nbr_off, *nbr;
    int nsteps;
};

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Bounded wait, by the 32 lanes of a warp together, until every CTA in
// nbr[j0 .. j1) has stored `target` steps (kWaitNs of device time, and
// independently 2^24 polls of one flag); true when they all have.
__device__ __noinline__ bool neighbours_done(const unsigned *flags, const int *nbr, int j0, int j1, unsigned target,
                                             int lane)
{
    const unsigned long long t0 = global_ns();
    for (int j = j0 + lane; j < j1; j += 32) {
        const unsigned *f = flags + (int64_t)nbr[j] * kRunFlagStride;
        int i = 0;
        while (ld_acquire_gpu(f) < target)
            if (++i > (1 << 24) || global_ns() - t0 > kWaitNs) return false;
    }
    return true;
}

// The fields of one sample that the rare slow paths read from global
// memory: its anatomy (p_w, p_g), its phi and face coefficients.
template <typename Real>
struct ItemCtx {
    const Real *pw, *pg, *phi_in, *H;  // pool order, block 0 of the sample
    int L;                             // log2 of the blocks per direction
};

// p_w, p_g of lab cell (x, y, z) of block blk: the interior or one face halo
template <typename Real>
__device__ __forceinline__ void pwpg_at(const ItemCtx<Real> &v, int blk, int x, int y, int z, Real &pw, Real &pg)
{
    const int L = v.L;
    int b = blk;
    if (x < 0) { b = nb_of(blk, L, 0); x += 8; }
    else if (x > 7) { b = nb_of(blk, L, 1); x -= 8; }
    else if (y < 0) { b = nb_of(blk, L, 2); y += 8; }
    else if (y > 7) { b = nb_of(blk, L, 3); y -= 8; }
    else if (z < 0) { b = nb_of(blk, L, 4); z += 8; }
    else if (z > 7) { b = nb_of(blk, L, 5); z -= 8; }
    const int64_t g = (int64_t)b * kBS3 + x + kBS * (y + kBS * z);
    pw = v.pw[g];
    pg = v.pg[g];
}

// Work source of one solve: the host-built block lists (heavy entries
// block * 4 + type, mixed blocks first; empty entries block).
template <typename Real>
struct PoolSource {
    static constexpr bool kSamples = false;  // one sample: rho and dt are constants
    const int *heavy, *empty;
    int nh, ne;
    const Real *phi_in;
    Real *phi_out;
    const Real *H, *pw, *pg;
    const unsigned short *meta;
    Real rho;
    double dt;
    int L, nblocks;
    unsigned *nan_flag;

    __device__ int total_heavy() const { return nh; }
    __device__ int total_empty() const { return ne; }
    __device__ void heavy_item(int g, int &p, int &e) const { p = 0; e = heavy[g]; }
    __device__ void empty_item(int g, int &p, int &e) const { p = 0; e = empty[g] * 4; }
    __device__ void params(int, double &r, double &d) const { r = (double)rho; d = dt; }
    __device__ const unsigned short *meta_of(int) const { return meta; }
    __device__ const Real *H_of(int) const { return H; }
    __device__ int64_t slot0(int) const { return 0; }
    __device__ ItemCtx<Real> ctx(int) const { return ItemCtx<Real>{pw, pg, phi_in, H, L}; }
    __device__ Real rho_of(int) const { return rho; }
    __device__ double dt_of(int) const { return dt; }
    __device__ unsigned *nan_of(int) const { return nan_flag; }
};

// Work source of a TMCMC batch step: the active samples (positions
// 0 .. nactive-1, longest horizon first); hpref / epref are prefix sums of
// the heavy / empty block counts over the positions, and the items of every
// position are decoded once per run (hdec, edec: global item g -> (position,
// entry)), so that the active ones are a prefix.  Sample p's pool starts at
// block p * nblocks of the phi buffers and of the face coefficients.
template <typename Real>
struct BatchSource {
    static constexpr bool kSamples = true;
    const int *hpref, *epref;
    const int *anatomy;     // per position
    int nactive;
    const Real *phi_in;
    Real *phi_out;
    const Real *H;          // all positions
    const Real *pw, *pg;    // all anatomies
    const unsigned short *meta;
    const Real *rho;        // per position
    const double *dt;       // per position
    int L, nblocks;
    unsigned *nan_flags;    // per position
    bool skip_empty;        // the empty blocks already hold their output

    __device__ int total_heavy() const { return hpref[nactive]; }
    __device__ int total_empty() const { return skip_empty ? 0 : epref[nactive]; }
    const int2 *hdec, *edec;
    __device__ void heavy_item(int g, int &p, int &e) const
    {
        const int2 d = hdec[g];
        p = d.x;
        e = d.y;
    }
    __device__ void empty_item(int g, int &p, int &e) const
    {
        const int2 d = edec[g];
        p = d.x;
        e = d.y;
    }
    __device__ void params(int p, double &r, double &d) const { r = (double)rho[p]; d = dt[p]; }
    __device__ const unsigned short *meta_of(int p) const { return meta + (int64_t)anatomy[p] * nblocks * kBS3; }
    __device__ const Real *H_of(int p) const { return H + (int64_t)p * nblocks * kFacesPerBlock; }
    __device__ int64_t slot0(int p) const { return (int64_t)p * nblocks; }
    __device__ ItemCtx<Real> ctx(int p) const
    {
        const int64_t a = (int64_t)anatomy[p] * nblocks * kBS3;
        return ItemCtx<Real>{pw + a, pg + a, phi_in + (int64_t)p * nblocks * kBS3, H_of(p), L};
    }
    __device__ Real rho_of(int p) const { return rho[p]; }
    __device__ double dt_of(int p) const { return dt[p]; }
    __device__ unsigned *nan_of(int p) const { return nan_flags + p; }
};

// The no-flux tests of a cell's six neighbours (x-, x+, y-, y+, z-, z+):
// low[k] = chf of neighbour k < 0.1, from its class bits in the meta word
// (kMixed) or, in a tissue block, knowing that every neighbour is kTissue.
// A kTissue neighbour with phi >= 0 has chf >= 0.1; so has one whose phi is
// NaN (the comparison is false), so with kClamped (phi_in holds the output
// of a step: +0 <= phi <= 1 or NaN) its test needs no evaluation.
template <typename Real, bool kMixed, bool kClamped, typename Source>
__device__ __forceinline__ void neighbour_low(const Source &src, int sp, int blk, int x, int y, int z, unsigned mw,
                                              const Real (&phn)[6], bool (&low)[6])
{
    const Real eps = (Real)0.1;
#pragma unroll
    for (int kk = 0; kk < 6; kk++) {
        bool slow;
        if (kMixed && ((mw >> (2 + kk)) & 1u)) {
            low[kk] = phn[kk] < eps;
            slow = false;
        } else {
            low[kk] = false;
            slow = (kMixed && ((mw >> (8 + kk)) & 1u)) || (!kClamped && !(phn[kk] >= (Real)0));
        }
        if (slow) {
            const int nx = x + (kk == 0 ? -1 : kk == 1 ? 1 : 0);
            const int ny = y + (kk == 2 ? -1 : kk == 3 ? 1 : 0);
            const int nz = z + (kk == 4 ? -1 : kk == 5 ? 1 : 0);
            Real pw, pg;
            pwpg_at(src.ctx(sp), blk, nx, ny, nz, pw, pg);
            low[kk] = domain_chf(phn[kk], pw, pg) < eps;
        }
    }
}

// The cells of one thread in a tissue (kMixed = false) or mixed block: its
// column (x, y) at z = z0 .. z0 + kCells - 1, everything from the stage.
// With kClamped a kTissue cell is inside the domain without a test (phi >= 0;
// a NaN phi yields NaN either way).  sp: the item's sample position, whose
// fields the rare slow paths read from global memory.
template <typename Real, int kCells, bool kMixed, bool kClamped, typename Source>
__device__ __forceinline__ void column_cells(const Source &src, int sp, const HeavySlot<Real> &S, int blk, int x,
                                             int y, int z0, int c0, Real rho, double ih2, double dt, int dt_finite,
                                             Real (&out)[kCells])
{
    const Real *in = S.in;
    Real p[kCells];
    unsigned mw[kCells];
#pragma unroll
    for (int i = 0; i < kCells; i++) {
        p[i] = in[c0 + 64 * i];
        mw[i] = kMixed ? (unsigned)S.meta[c0 + 64 * i] : kMetaAllTissue;
    }
#pragma unroll
    for (int i = 0; i < kCells; i++) {
        const Real phi = p[i];
        const int z = z0 + i, c = c0 + 64 * i;
        const unsigned cls = mw[i] & 3u;
        bool dom;
        if (cls == kTissue && (kClamped || phi >= (Real)0)) dom = true;
        else if (cls == kEmpty) dom = phi > (Real)0;
        else {
            Real pw, pg;
            pwpg_at(src.ctx(sp), blk, x, y, z, pw, pg);
            dom = in_domain(pw, pg, phi);
        }
        if (!dom) {
            out[i] = dt_finite ? clamp01(phi) : cell_update(phi, (Real)0., dt);
            continue;
        }
        // one shared load per neighbour: interior or face halo by address
        Real phn[6];
        phn[0] = *(x > 0 ? &in[c - 1] : &S.xm[(z * 8 + y) * 4 + 3]);
        phn[1] = *(x < 7 ? &in[c + 1] : &S.xp[(z * 8 + y) * 4]);
        phn[2] = *(y > 0 ? &in[c - 8] : &S.ym[z * 8 + x]);
        phn[3] = *(y < 7 ? &in[c + 8] : &S.yp[z * 8 + x]);
        phn[4] = i > 0 ? p[i - 1] : *(z > 0 ? &in[c - 64] : &S.zm[y * 8 + x]);
        phn[5] = i < kCells - 1 ? p[i + 1] : *(z < 7 ? &in[c + 64] : &S.zp[y * 8 + x]);
        const int rx = (z * 8 + y) * 9 + x, ry = 576 + (z * 9 + y) * 8 + x, rz = 1152 + (z * 8 + y) * 8 + x;
        bool low[6];
        if (!kMixed && (kClamped || (phn[0] >= (Real)0 && phn[1] >= (Real)0 && phn[2] >= (Real)0 &&
                                     phn[3] >= (Real)0 && phn[4] >= (Real)0 && phn[5] >= (Real)0))) {
            // kTissue neighbours with phi >= 0: chf >= 0.1, no doubling
#pragma unroll
            for (int kk = 0; kk < 6; kk++) low[kk] = false;
        } else {
            neighbour_low<Real, kMixed, kClamped>(src, sp, blk, x, y, z, mw[i], phn, low);
        }
        const Real dphidt = cell_rhs_flags<Real>(S.H[rx], S.H[rx + 1], S.H[ry], S.H[ry + 8], S.H[rz], S.H[rz + 64],
                                                 low, phn, phi, rho, ih2);
        out[i] = cell_update(phi, dphidt, dt);
    }
}

// A cell of an empty block (every cell and face-halo cell kEmpty) with
// phi > 0: inside the domain, neighbours and coefficients from global memory.
template <typename Real>
__device__ __noinline__ Real empty_cell(const ItemCtx<Real> v, int blk, int c, Real phi, Real rho, double ih2,
                                        double dt, int dt_finite)
{
    const Real *phi_in = v.phi_in, *H = v.H;
    if (!(phi > (Real)0)) return dt_finite ? clamp01(phi) : cell_update(phi, (Real)0., dt);
    const int L = v.L;
    const int x = c & 7, y = (c >> 3) & 7, z = c >> 6;
    // loads cached in L2 only: in a run of steps the buffer is rewritten
    // between two of its reads by other CTAs
    const Real *b0 = phi_in + (int64_t)blk * kBS3;
    Real phn[6];
    phn[0] = __ldcg(x > 0 ? &b0[c - 1] : &phi_in[(int64_t)nb_of(blk, L, 0) * kBS3 + c + 7]);
    phn[1] = __ldcg(x < 7 ? &b0[c + 1] : &phi_in[(int64_t)nb_of(blk, L, 1) * kBS3 + c - 7]);
    phn[2] = __ldcg(y > 0 ? &b0[c - 8] : &phi_in[(int64_t)nb_of(blk, L, 2) * kBS3 + c + 56]);
    phn[3] = __ldcg(y < 7 ? &b0[c + 8] : &phi_in[(int64_t)nb_of(blk, L, 3) * kBS3 + c - 56]);
    phn[4] = __ldcg(z > 0 ? &b0[c - 64] : &phi_in[(int64_t)nb_of(blk, L, 4) * kBS3 + c + 448]);
    phn[5] = __ldcg(z < 7 ? &b0[c + 64] : &phi_in[(int64_t)nb_of(blk, L, 5) * kBS3 + c - 448]);
    const Real eps = (Real)0.1;
    bool low[6];
#pragma unroll
    for (int kk = 0; kk < 6; kk++) low[kk] = phn[kk] < eps;
    const Real *Hb = H + (int64_t)blk * kFacesPerBlock;
    const int rx = (z * 8 + y) * 9 + x, ry = 576 + (z * 9 + y) * 8 + x, rz = 1152 + (z * 8 + y) * 8 + x;
    const Real dphidt =
        cell_rhs_flags<Real>(Hb[rx], Hb[rx + 1], Hb[ry], Hb[ry + 8], Hb[rz], Hb[rz + 64], low, phn, phi, rho, ih2);
    return cell_update(phi, dphidt, dt);
}

// OR of the bit patterns: zero exactly when every value is +0.0
__device__ __forceinline__ unsigned bits_or(float a) { return __float_as_uint(a); }
__device__ __forceinline__ unsigned bits_or(double a)
{
    const unsigned long long b = (unsigned long long)__double_as_longlong(a);
    return (unsigned)b | (unsigned)(b >> 32);
}

// resident CTAs per SM the register allocation targets: what the shared
// memory of the default shapes allows (FP32 4, FP64 3)
#ifndef GBFK_TMA_MIN_BLOCKS_F32
#define GBFK_TMA_MIN_BLOCKS_F32 4
#endif
#ifndef GBFK_TMA_MIN_BLOCKS_F64
#define GBFK_TMA_MIN_BLOCKS_F64 3
#endif

// kMulti: a run of run.nsteps steps in one cooperative launch (one pool, and
// kClamped: every input of the run is the output of a step).  Each CTA keeps
// its items for the whole run; after its consumers have stored step s, one
// of them arrives on a grid barrier (a counter in global memory, waits
// bounded like every other) and then releases the producer to issue step
// s + 1, whose copies read what every CTA wrote in step s.  The step
// arithmetic is the one-step kernel's: a run of n steps gives the bits of n
// launches.
template <typename Real, int kWarps, int kHeavySlots, int kEmptySlots, bool kClamped, bool kMulti, typename Source>
__global__ void __launch_bounds__((kWarps + 1) * 32, kWarps == 8 ? (sizeof(Real) == 4 ? GBFK_TMA_MIN_BLOCKS_F32
                                                                                       : GBFK_TMA_MIN_BLOCKS_F64)
                                                                  : 1)
rd_step_tma_kernel(const Source src, double ih2, unsigned *err_flag, const StepRun<Real> run,
                   const __grid_constant__ TmaMaps<kMulti ? 3 : 1> maps)
{
    // Programmatic dependent launch: a step launched with it may be scheduled
    // while the previous grid on the stream still runs.  It lets the next
    // step's grid be scheduled as this one's CTAs finish, stages its work
    // items (host-written lists, complete before any later kernel starts) and
    // sets up its barriers, and only then waits until the previous grid has
    // completed and its writes are visible, before any other global access.
    // Without the launch attribute both instructions return at once.
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    using Lay = SmemLayout<Real, kHeavySlots, kEmptySlots>;
    constexpr int kThreads = kWarps * 32;  // consumer threads
    constexpr int kCells = kBS3 / kThreads;
    static_assert(kCells * kThreads == kBS3 && kCells >= 1 && kCells <= 8, "consumer warps per block");
    static_assert(kEmptySlots % kWarps == 0, "an empty slot must serve one warp");
    static_assert(!kMulti || (kClamped && !Source::kSamples), "a run of steps: one pool, clamped inputs");
    constexpr int kVec = 16 / sizeof(Real);       // cells per 16-byte vector
    constexpr int kOwnVecs = kBS3 / (32 * kVec);  // vectors per lane of an empty block's warp
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ unsigned run_abort;  // kMulti: a grid barrier wait gave up
    HeavySlot<Real> *heavy = reinterpret_cast<HeavySlot<Real> *>(smem + Lay::heavy);
    Real *empties = reinterpret_cast<Real *>(smem + Lay::empty);
    uint64_t *hfull = reinterpret_cast<uint64_t *>(smem + Lay::bars);
    uint64_t *hfree = hfull + kHeavySlots;
    uint64_t *efull = hfree + kHeavySlots;
    uint64_t *efree = efull + kEmptySlots;
    uint64_t *go = efree + kEmptySlots;  // kMulti, per step boundary: the producer may issue the next step
    uint64_t *done = go + 1;             // kMulti, per step boundary: every consumer warp has stored the step
    SlotHdr *hhdr = reinterpret_cast<SlotHdr *>(smem + Lay::hdr);
    SlotHdr *ehdr = hhdr + kHeavySlots;
    const int t = threadIdx.x;
    const int c = blockIdx.x, G = gridDim.x;
    const int nsteps = kMulti ? run.nsteps : 1;
    const int NH = src.total_heavy(), NE = src.total_empty();
    const int nh = NH > c ? (NH - 1 - c) / G + 1 : 0;
    // empty items: one pool counts them from the other end (CTA c takes
    // G - 1 - c, 2G - 1 - c, ...), so that the CTAs that get one more heavy
    // item than others get no more empty ones; a batch: c, c + G, ...
    const int ce = Source::kSamples ? c : G - 1 - c;
    const int ne = NE > ce ? (NE - 1 - ce) / G + 1 : 0;
    if (!kMulti && nh + ne == 0) return;  // uniform across the CTA (a run's CTAs all take the barriers)
    // one pool: the CTA's items staged in shared memory, issued by lane 0
    // alone; a batch: decoded 32 at a time by the producer warp
    constexpr bool kStaged = !Source::kSamples;
    int *items = reinterpret_cast<int *>(smem + Lay::items);
    if (kStaged) {
        if (nh + ne > kMaxItems) {  // the launcher keeps nh + ne in range
            if (t == 0) atomicOr(err_flag, 2u);
            return;
        }
        int unused;
        for (int i = t; i < nh; i += blockDim.x) src.heavy_item(c + i * G, unused, items[i]);
        for (int i = t; i < ne; i += blockDim.x) src.empty_item(ce + i * G, unused, items[nh + i]);
    }
    if (t == 0) {
        for (int i = 0; i < kHeavySlots; i++) {
            mbar_init(&hfull[i], 1);
            mbar_init(&hfree[i], kWarps);
        }
        for (int i = 0; i < kEmptySlots; i++) {
            mbar_init(&efull[i], 1);
            mbar_init(&efree[i], 1);
        }
        if (kMulti) {
            mbar_init(go, 1);
            mbar_init(done, kWarps);
            run_abort = 0;
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();  // the only CTA-wide barrier
    asm volatile("griddepcontrol.wait;" ::: "memory");

    // the buffers and tensor maps of step s
    auto in_of = [&](int s) -> const Real * {
        if (!kMulti) return src.phi_in;
        return s == 0 ? run.in0 : run.buf[(s - 1) & 1];
    };
    auto out_of = [&](int s) -> Real * {
        if (!kMulti) return src.phi_out;
        return s == nsteps - 1 ? run.last : run.buf[s & 1];
    };
    auto maps_of = [&](int s) -> const TmaMapSet & { return maps.b[kMulti ? (s == 0 ? 0 : 1 + ((s - 1) & 1)) : 0]; };

    const int L = src.L;
    const int lane = t & 31;
    if (t >= kThreads) {
        // producer warp; lane 0 puts an item in flight in slot s
        auto issue_heavy = [&](int s, int p, int e, double irho, double idt, const Real *in, const TmaMapSet &ms) {
            const int blk = e >> 2, bt = e & 3;
            const int64_t s0 = src.slot0(p);
            if (Source::kSamples) {
                hhdr[s].dt = idt;
                hhdr[s].rho = irho;
                hhdr[s].p = p;
            }
            hhdr[s].e = e;
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            HeavySlot<Real> &S = heavy[s];
            uint64_t *bar = &hfull[s];
            uint32_t bytes = (kBS3 + 2 * 256 + 4 * 64 + kFacesPerBlock) * sizeof(Real);
            if (bt == kBlockMixed) bytes += kBS3 * sizeof(unsigned short);
            mbar_arrive_expect_tx(bar, bytes);
            bulk_g2s(S.in, in + (s0 + blk) * kBS3, kBS3 * sizeof(Real), bar);
            box_g2s(S.xm, &ms.m[0], 4, 0, 0, (int)(s0 + nb_of(blk, L, 0)), bar);
            box_g2s(S.xp, &ms.m[0], 0, 0, 0, (int)(s0 + nb_of(blk, L, 1)), bar);
            box_g2s(S.ym, &ms.m[1], 0, 7, 0, (int)(s0 + nb_of(blk, L, 2)), bar);
            box_g2s(S.yp, &ms.m[1], 0, 0, 0, (int)(s0 + nb_of(blk, L, 3)), bar);
            box_g2s(S.zm, &ms.m[2], 0, 0, 7, (int)(s0 + nb_of(blk, L, 4)), bar);
            box_g2s(S.zp, &ms.m[2], 0, 0, 0, (int)(s0 + nb_of(blk, L, 5)), bar);
            bulk_g2s(S.H, src.H_of(p) + (int64_t)blk * kFacesPerBlock, kFacesPerBlock * sizeof(Real), bar);
            if (bt == kBlockMixed)
                bulk_g2s(S.meta, src.meta_of(p) + (int64_t)blk * kBS3, kBS3 * sizeof(unsigned short), bar);
        };
        auto issue_empty = [&](int s, int p, int e, double irho, double idt, const Real *in) {
            if (Source::kSamples) {
                ehdr[s].dt = idt;
                ehdr[s].rho = irho;
                ehdr[s].p = p;
            }
            ehdr[s].e = e;
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_arrive_expect_tx(&efull[s], kBS3 * sizeof(Real));
            bulk_g2s(empties + s * kBS3, in + (src.slot0(p) + (e >> 2)) * kBS3, kBS3 * sizeof(Real), &efull[s]);
        };
        int jh = 0, je = 0;  // items issued, over all steps of a run
        bool ok = true;
        unsigned site = 0;  // which wait gave up (error word bits 5..7)
        if (kStaged) {
            if (!kMulti && lane != 0) return;
            for (int st = 0; st < nsteps && ok; st++) {
                if (kMulti && st > 0) {
                    // this CTA's consumers have stored step st - 1 (go), and
                    // so have the CTAs that own the face neighbours of its
                    // blocks: the inputs of step st are complete, and no
                    // block that step st overwrites is still read
                    bool w = mbar_wait(go, (st - 1) & 1) && !*(volatile unsigned *)&run_abort;
                    if (w) w = neighbours_done(run.flags, run.nbr, run.nbr_off[c], run.nbr_off[c + 1], (unsigned)st, lane);
                    if (!__all_sync(0xffffffffu, w)) {
                        ok = false;
                        site = 128u;
                        break;
                    }
                    __syncwarp();
                    if (lane == 0) asm volatile("fence.proxy.async.global;" ::: "memory");
                }
                const Real *in = in_of(st);
                const TmaMapSet &ms = maps_of(st);
                if (lane == 0) {
                    int lh = 0, le = 0;  // items of this step
                    while (lh < nh || le < ne) {
                        if (heavy_next(lh, le, nh, ne)) {
                            const int s = jh % kHeavySlots;
                            if (jh >= kHeavySlots && !mbar_wait(&hfree[s], ((jh / kHeavySlots) - 1) & 1)) {
                                ok = false;
                                site = 32u;
                                break;
                            }
                            issue_heavy(s, 0, items[lh], 0., 0., in, ms);
                            lh++;
                            jh++;
                        } else {
                            const int s = je % kEmptySlots;
                            if (je >= kEmptySlots && !mbar_wait(&efree[s], ((je / kEmptySlots) - 1) & 1)) {
                                ok = false;
                                site = 64u;
                                break;
                            }
                            issue_empty(s, 0, items[nh + le], 0., 0., in);
                            le++;
                            je++;
                        }
                    }
                }
                if (kMulti) ok = __shfl_sync(0xffffffffu, ok, 0);
            }
        } else {
            // the lanes decode 32 items of each kind at a time, lane 0 issues them
            const Real *in = in_of(0);
            const TmaMapSet &ms = maps_of(0);
            int hbase = 0, ebase = 0;
            int hp = 0, he = 0, ep = 0, ee = 0;
            double hrho = 0, hdt = 0, erho = 0, edt = 0;
            if (lane < nh) {
                src.heavy_item(c + lane * G, hp, he);
                src.params(hp, hrho, hdt);
            }
            if (lane < ne) {
                src.empty_item(c + lane * G, ep, ee);
                src.params(ep, erho, edt);
            }
            while (jh < nh || je < ne) {
                if (heavy_next(jh, je, nh, ne)) {
                    if (jh == hbase + 32) {
                        hbase = jh;
                        if (jh + lane < nh) {
                            src.heavy_item(c + (jh + lane) * G, hp, he);
                            src.params(hp, hrho, hdt);
                        }
                    }
                    const int k = jh - hbase;
                    const int e = __shfl_sync(0xffffffffu, he, k), p = __shfl_sync(0xffffffffu, hp, k);
                    const double irho = __shfl_sync(0xffffffffu, hrho, k), idt = __shfl_sync(0xffffffffu, hdt, k);
                    const int s = jh % kHeavySlots;
                    bool w = true;
                    if (lane == 0 && jh >= kHeavySlots) w = mbar_wait(&hfree[s], ((jh / kHeavySlots) - 1) & 1);
                    if (!__shfl_sync(0xffffffffu, w, 0)) {
                        ok = false;
                        site = 32u;
                        break;
                    }
                    if (lane == 0) issue_heavy(s, p, e, irho, idt, in, ms);
                    jh++;
                } else {
                    if (je == ebase + 32) {
                        ebase = je;
                        if (je + lane < ne) {
                            src.empty_item(c + (je + lane) * G, ep, ee);
                            src.params(ep, erho, edt);
                        }
                    }
                    const int k = je - ebase;
                    const int e = __shfl_sync(0xffffffffu, ee, k), p = __shfl_sync(0xffffffffu, ep, k);
                    const double irho = __shfl_sync(0xffffffffu, erho, k), idt = __shfl_sync(0xffffffffu, edt, k);
                    const int s = je % kEmptySlots;
                    bool w = true;
                    if (lane == 0 && je >= kEmptySlots) w = mbar_wait(&efree[s], ((je / kEmptySlots) - 1) & 1);
                    if (!__shfl_sync(0xffffffffu, w, 0)) {
                        ok = false;
                        site = 64u;
                        break;
                    }
                    if (lane == 0) issue_empty(s, p, e, irho, idt, in);
                    je++;
                }
            }
        }
        if (lane == 0) {
            if (!ok) atomicOr(err_flag, 1u | site);
            // the CTA's shared memory must outlive every copy in flight (bounded)
            for (int j = jh - kHeavySlots > 0 ? jh - kHeavySlots : 0; j < jh; j++)
                mbar_wait(&hfull[j % kHeavySlots], (j / kHeavySlots) & 1);
            for (int j = je - kEmptySlots > 0 ? je - kEmptySlots : 0; j < je; j++)
                mbar_wait(&efull[j % kEmptySlots], (j / kEmptySlots) & 1);
        }
        return;
    }

    const int warp = t >> 5;
    const int x = t & 7, y = (t >> 3) & 7, z0 = (t >> 6) * kCells;
    const int c0 = x + kBS * (y + kBS * z0);
    // items over all steps of a run: heavy item jh of step st is item
    // st * nh + jh, empty item je of step st is st * ne + je; a warp takes the
    // empty items whose run index is warp mod kWarps, so each empty slot
    // keeps serving one warp
    int next_e = warp;  // this warp's next empty item (run index)
    for (int st = 0; st < nsteps; st++) {
        const Real *in = in_of(st);
        Real *out = out_of(st);
        int jh = 0, je = next_e - st * ne;  // next heavy item; next empty item of this warp (this step)
        while (jh < nh || je < ne) {
            if (heavy_next(jh, je, nh, ne)) {
                const int J = st * nh + jh;
                const int s = J % kHeavySlots;
                if (!__all_sync(0xffffffffu, mbar_wait(&hfull[s], (J / kHeavySlots) & 1))) {
                    if (lane == 0) atomicOr(err_flag, 1u | 8u);
                    return;
                }
                const int e = hhdr[s].e, blk = e >> 2;
                int p = 0;
                double dt;
                Real rho;
                if (Source::kSamples) {
                    p = hhdr[s].p;
                    dt = hhdr[s].dt;
                    rho = (Real)hhdr[s].rho;
                } else {
                    dt = src.dt_of(0);
                    rho = src.rho_of(0);
                }
                Real o[kCells];
                if ((e & 3) == kBlockTissue)
                    column_cells<Real, kCells, false, kClamped>(src, p, heavy[s], blk, x, y, z0, c0, rho, ih2, dt,
                                                                isfinite(dt), o);
                else
                    column_cells<Real, kCells, true, kClamped>(src, p, heavy[s], blk, x, y, z0, c0, rho, ih2, dt,
                                                               isfinite(dt), o);
                // every shared read of this warp is done: release the slot
                __syncwarp();
                if (lane == 0) mbar_arrive(&hfree[s], 1);
                Real *ob = out + (src.slot0(p) + blk) * kBS3;
                bool bad = false;
#pragma unroll
                for (int i = 0; i < kCells; i++) {
                    bad |= (o[i] != o[i]);
                    ob[c0 + 64 * i] = o[i];
                }
                if (bad) atomicOr(src.nan_of(p), 1u);
                jh++;
                continue;
            }
            const int j = je;
            je += kWarps;
            const int J = st * ne + j;
            const int s = J % kEmptySlots;
            if (!__all_sync(0xffffffffu, mbar_wait(&efull[s], (J / kEmptySlots) & 1))) {
                if (lane == 0) atomicOr(err_flag, 1u | 16u);
                return;
            }
            const Real *ein = empties + s * kBS3;
            const int blk = ehdr[s].e >> 2;
            const int p = Source::kSamples ? ehdr[s].p : 0;
            Real *ob = out + (src.slot0(p) + blk) * kBS3;
            Real pv[kOwnVecs][kVec];
            unsigned bits = 0;
#pragma unroll
            for (int q = 0; q < kOwnVecs; q++) {
                vec_lds<Real, kVec>(ein + (q * 32 + lane) * kVec, pv[q]);
#pragma unroll
                for (int i = 0; i < kVec; i++) bits |= bits_or(pv[q][i]);
            }
            if (bits == 0) {
                // every cell +0.0: outside the domain, and the clamp leaves +0.0
                __syncwarp();
                if (lane == 0) mbar_arrive(&efree[s], 1);
#pragma unroll
                for (int q = 0; q < kOwnVecs; q++) vec_stg<Real, kVec>(ob + (q * 32 + lane) * kVec, pv[q]);
                continue;
            }
            const double dt = Source::kSamples ? ehdr[s].dt : src.dt_of(0);
            const int dt_finite = isfinite(dt);
            bool any = false, bad = false;
#pragma unroll
            for (int q = 0; q < kOwnVecs; q++)
#pragma unroll
                for (int i = 0; i < kVec; i++) any |= pv[q][i] > (Real)0;  // the domain test of a kEmpty cell
            if (any) {
                // tumour outside the anatomy: an empty block's slot holds no halo
                // or coefficients, read them from global memory (rare)
                ItemCtx<Real> cx = src.ctx(p);
                cx.phi_in = in + src.slot0(p) * kBS3;
                const Real rho = Source::kSamples ? (Real)ehdr[s].rho : src.rho_of(0);
#pragma unroll 1
                for (int q = 0; q < kOwnVecs * kVec; q++) {
                    const int cc = ((q / kVec) * 32 + lane) * kVec + q % kVec;
                    const Real o = empty_cell(cx, blk, cc, ein[cc], rho, ih2, dt, dt_finite);
                    bad |= (o != o);
                    ob[cc] = o;
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(&efree[s], 1);
            } else {
                __syncwarp();
                if (lane == 0) mbar_arrive(&efree[s], 1);
#pragma unroll
                for (int q = 0; q < kOwnVecs; q++) {
                    Real o[kVec];
#pragma unroll
                    for (int i = 0; i < kVec; i++) {
                        o[i] = dt_finite ? clamp01(pv[q][i]) : cell_update(pv[q][i], (Real)0., dt);
                        bad |= (o[i] != o[i]);
                    }
                    vec_stg<Real, kVec>(ob + (q * 32 + lane) * kVec, o);
                }
            }
            if (bad) atomicOr(src.nan_of(p), 1u);
        }
        next_e = st * ne + je;
        if (kMulti && st + 1 < nsteps) {
            // step boundary: each warp reports its stores of step st; thread 0
            // waits for all of them (bounded: a warp that gave up never
            // arrives), publishes this CTA's step count to the CTAs that
            // read its blocks, and opens step st + 1 to the producer and to
            // every consumer warp.  All warps wait for that: a warp with no
            // item in step st + 1 would otherwise report step st + 1 before
            // this boundary has passed.
            __syncwarp();
            if (lane == 0) mbar_arrive(done, 1);
            if (t == 0) {
                if (mbar_wait(done, st & 1)) {
                    // the stores, then the flag; the TMA copies of the next
                    // step (async proxy) read what the generic stores wrote
                    asm volatile("fence.proxy.async.global;" ::: "memory");
                    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(run.flags + (int64_t)c * kRunFlagStride),
                                 "r"((unsigned)(st + 1))
                                 : "memory");
                } else {
                    atomicOr(err_flag, 256u);
                    run_abort = 1;
                }
                mbar_arrive(go, 1);
            }
            const bool opened = __all_sync(0xffffffffu, mbar_wait(go, st & 1));
            if (!opened || *(volatile unsigned *)&run_abort) {
                if (!opened && lane == 0) atomicOr(err_flag, 1u | 128u);
                return;
            }
        }
    }
}

typedef CUresult (*EncodeTiled)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_fn()
{
    static std::once_flag once;
    static EncodeTiled fn = nullptr;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiled>(p);
    });
    return fn;
}

// One launch shape: consumer warps per CTA and slots of the two rings.
template <typename Real, int kWarps, int kHeavySlots, int kEmptySlots>
struct Shape {
    static constexpr int kThreads = (kWarps + 1) * 32;
    static constexpr size_t kSmem = SmemLayout<Real, kHeavySlots, kEmptySlots>::bytes;

    // resident CTAs on this part for the kernels of one work source (kMulti:
    // the run kernel), taken once per process
    template <typename Source, bool kMulti = false>
    static cudaError_t grid(int &g)
    {
        static int cached = 0;
        static std::mutex mu;
        std::lock_guard<std::mutex> lk(mu);
        if (!cached) {
            cudaError_t e;
            int per_sm = 0;
            if constexpr (kMulti) {
                auto k = rd_step_tma_kernel<Real, kWarps, kHeavySlots, kEmptySlots, true, true, Source>;
                if ((e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem)) !=
                    cudaSuccess)
                    return e;
                if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kThreads, kSmem)) != cudaSuccess)
                    return e;
            } else {
                auto k = rd_step_tma_kernel<Real, kWarps, kHeavySlots, kEmptySlots, false, false, Source>;
                auto kc = rd_step_tma_kernel<Real, kWarps, kHeavySlots, kEmptySlots, true, false, Source>;
                if ((e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem)) !=
                    cudaSuccess)
                    return e;
                if ((e = cudaFuncSetAttribute(kc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem)) !=
                    cudaSuccess)
                    return e;
                if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kThreads, kSmem)) != cudaSuccess)
                    return e;
            }
            int dev = 0, sms = 0;
            if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
            if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
            if (kMulti && per_sm < 1) return cudaErrorCooperativeLaunchTooLarge;
            cached = sms * (per_sm > 0 ? per_sm : 1);
        }
        g = cached;
        return cudaSuccess;
    }

    template <typename Source>
    static cudaError_t launch(const Source &src, int items, double ih2, bool clamped, unsigned *err_flag,
                              const CUtensorMap *maps, cudaStream_t s)
    {
        int g = 0;
        cudaError_t e = grid<Source>(g);
        if (e != cudaSuccess) return e;
        const int nctas = items < g ? items : g;
        auto k = clamped ? rd_step_tma_kernel<Real, kWarps, kHeavySlots, kEmptySlots, true, false, Source>
                         : rd_step_tma_kernel<Real, kWarps, kHeavySlots, kEmptySlots, false, false, Source>;
        TmaMaps<1> m;
        for (int i = 0; i < 3; i++) m.b[0].m[i] = maps[i];
        const StepRun<Real> run = {};
        // one pool: launched with programmatic dependent launch, so that the
        // next step's launch overlaps this step's tail
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(nctas);
        cfg.blockDim = dim3(kThreads);
        cfg.dynamicSmemBytes = kSmem;
        cfg.stream = s;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = Source::kSamples ? 0 : 1;
        return cudaLaunchKernelEx(&cfg, k, src, ih2, err_flag, run, m);
    }

    // CTAs of a run over `items` blocks: all that fit (GBFK_RUN_CTAS_PER_SM,
    // a tuning knob, asks for fewer per SM)
    static cudaError_t run_grid(int items, int &nctas)
    {
        int g = 0;
        cudaError_t e = grid<PoolSource<Real>, true>(g);
        if (e != cudaSuccess) return e;
        static const int per_sm = [] {
            const char *v = getenv("GBFK_RUN_CTAS_PER_SM");
            return v ? atoi(v) : 0;
        }();
        if (per_sm > 0) {
            int dev = 0, sms = 0;
            if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
            if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
            if (sms * per_sm < g) g = sms * per_sm;
        }
        if ((int64_t)items > (int64_t)g * (kMaxItems - 2)) return cudaErrorInvalidValue;
        nctas = items < g ? items : g;
        return cudaSuccess;
    }

    // a run of steps of one pool in one cooperative launch (every CTA
    // resident: a CTA waits for the CTAs of its neighbours); the step flags
    // are zeroed first
    static cudaError_t launch_run(const PoolSource<Real> &src, int items, int ctas, double ih2, unsigned *err_flag,
                                  const StepRun<Real> &run, const TmaMaps<3> &maps, cudaStream_t s)
    {
        int nctas = 0;
        cudaError_t e = run_grid(items, nctas);
        if (e != cudaSuccess) return e;
        if (nctas != ctas) return cudaErrorInvalidValue;  // the neighbour lists were made for `ctas` CTAs
        if ((e = cudaMemsetAsync(run.flags, 0, (size_t)nctas * kRunFlagStride * sizeof(unsigned), s)) != cudaSuccess)
            return e;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(nctas);
        cfg.blockDim = dim3(kThreads);
        cfg.dynamicSmemBytes = kSmem;
        cfg.stream = s;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        return cudaLaunchKernelEx(&cfg, rd_step_tma_kernel<Real, kWarps, kHeavySlots, kEmptySlots, true, true,
                                                           PoolSource<Real>>,
                                  src, ih2, err_flag, run, maps);
    }
};

// launch shape from GBFK_TMA_SHAPE="consumer warps,heavy slots,empty slots"
// (a tuning knob), else -1: the default of the Real type (8 warps and 8
// empty slots; 2 heavy slots in FP32, 1 in FP64: fastest at 256^3)
int tma_shape_code()
{
    static int code = -1;
    static std::once_flag once;
    std::call_once(once, [] {
        if (const char *e = getenv("GBFK_TMA_SHAPE")) {
            int w = 0, hv = 0, em = 0;
            if (sscanf(e, "%d,%d,%d", &w, &hv, &em) == 3) code = (w * 10 + hv) * 100 + em;
        }
    });
    return code;
}

#define GBFK_TMA_SHAPES(X) \
    X(8, 2, 8)             \
    X(8, 3, 8)             \
    X(8, 2, 16)            \
    X(8, 1, 8)             \
    X(4, 2, 8)             \
    X(16, 2, 16)

// the shape of a code (consumer warps * 1000 + heavy slots * 100 + empty
// slots), or the default for any code not in the list
template <typename Real, typename F>
cudaError_t with_shape_code(int code, F &&f)
{
#define GBFK_TMA_CASE(W, HV, EM) \
    case (W * 10 + HV) * 100 + EM: return f(Shape<Real, W, HV, EM>());
    switch (code) {
        GBFK_TMA_SHAPES(GBFK_TMA_CASE)
    default:
        if constexpr (sizeof(Real) == 4) return f(Shape<Real, 8, 2, 8>());
        else return f(Shape<Real, 8, 1, 8>());
    }
#undef GBFK_TMA_CASE
}

template <typename Real, typename F>
cudaError_t with_shape(F &&f)
{
    return with_shape_code<Real>(tma_shape_code(), f);
}

}  // namespace

// Tensor maps of a pool buffer of `nslots` 8^3 blocks viewed as
// [slot][z][y][x]: maps[0] the x-face box (4 x 8 x 8), maps[1] the y-face box
// (8 x 1 x 8), maps[2] the z-face box (8 x 8 x 1).
cudaError_t make_pool_tensor_maps(void *base, int nslots, int real_bytes, CUtensorMap maps[3])
{
    EncodeTiled enc = encode_fn();
    if (!enc) return cudaErrorNotSupported;
    const cuuint64_t es = (cuuint64_t)real_bytes;
    const cuuint64_t dims[4] = {8, 8, 8, (cuuint64_t)nslots};
    const cuuint64_t strides[3] = {8 * es, 64 * es, 512 * es};
    const cuuint32_t boxes[3][4] = {{4, 8, 8, 1}, {8, 1, 8, 1}, {8, 8, 1, 1}};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUtensorMapDataType dt = real_bytes == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    for (int i = 0; i < 3; i++) {
        if (enc(&maps[i], dt, 4, base, dims, strides, boxes[i], estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return cudaErrorInvalidValue;
    }
    return cudaSuccess;
}

// Whether the pipelined step applies to a view: a uniform periodic 2^L grid
// in slots 0..n-1 whose items fit each CTA's staging buffer.
template <typename Real>
bool tma_step_eligible(const PoolView<Real> &v)
{
    if (v.log2_bpd < 0 || !v.identity_slots || v.nblocks <= 0) return false;
    int g = 0;
    if (with_shape<Real>([&](auto sh) { return decltype(sh)::template grid<PoolSource<Real>>(g); }) != cudaSuccess)
        return false;
    return (int64_t)v.nblocks <= (int64_t)g * (kMaxItems - 2);
}

template <typename Real>
cudaError_t launch_rd_step_tma(const PoolView<Real> &v, const BlockLists &lists, const Real *H,
                               const unsigned short *meta, double ih2, const Real *phi_in, bool clamped,
                               Real *phi_out, Real rho, double dt, unsigned *nan_flag, unsigned *err_flag,
                               const CUtensorMap *maps, bool skip_empty, cudaStream_t s)
{
    if (lists.n_heavy + lists.n_empty <= 0) return cudaSuccess;
    if (!tma_step_eligible(v) || lists.n_heavy + lists.n_empty != v.nblocks) return cudaErrorInvalidValue;
    if (skip_empty && lists.n_heavy <= 0) return cudaSuccess;
    PoolSource<Real> src;
    src.heavy = lists.heavy;
    src.empty = lists.empty;
    src.nh = lists.n_heavy;
    src.ne = skip_empty ? 0 : lists.n_empty;
    src.phi_in = phi_in;
    src.phi_out = phi_out;
    src.H = H;
    src.pw = v.pw;
    src.pg = v.pg;
    src.meta = meta;
    src.rho = rho;
    src.dt = dt;
    src.L = v.log2_bpd;
    src.nblocks = v.nblocks;
    src.nan_flag = nan_flag;
    const int items = src.nh + src.ne;
    return with_shape<Real>([&](auto sh) {
        return decltype(sh)::template launch<PoolSource<Real>>(src, items, ih2, clamped, err_flag, maps, s);
    });
}

// The CTAs of a run over a grid's step lists, and per CTA the other CTAs
// that own a face neighbour of one of its blocks (CSR).  CTA c of G owns
// heavy items c, c + G, ... and empty items G - 1 - c, 2G - 1 - c, ... (the
// kernel's assignment).
template <typename Real>
cudaError_t rd_run_layout(const PoolView<Real> &v, const int *heavy, int n_heavy, const int *empty, int n_empty,
                          int &ctas, std::vector<int> &nbr_off, std::vector<int> &nbr)
{
    const int nb = n_heavy + n_empty;
    if (nb != v.nblocks || v.log2_bpd < 0) return cudaErrorInvalidValue;
    int G = 0;
    cudaError_t e = with_shape<Real>([&](auto sh) { return decltype(sh)::run_grid(nb, G); });
    if (e != cudaSuccess) return e;
    std::vector<int> owner(nb, -1);
    for (int g = 0; g < n_heavy; g++) owner[heavy[g] >> 2] = g % G;
    for (int g = 0; g < n_empty; g++) owner[empty[g]] = G - 1 - g % G;
    for (int b = 0; b < nb; b++)
        if (owner[b] < 0) return cudaErrorInvalidValue;
    std::vector<std::vector<int>> sets(G);
    const int L = v.log2_bpd, m = (1 << L) - 1;
    for (int b = 0; b < nb; b++) {
        const int bx = b & m, by = (b >> L) & m, bz = b >> (2 * L);
        for (int f = 0; f < 6; f++) {
            int x = bx, y = by, z = bz;
            const int d = f >> 1, sg = (f & 1) ? 1 : -1;
            if (d == 0) x = (x + sg) & m;
            else if (d == 1) y = (y + sg) & m;
            else z = (z + sg) & m;
            const int o = owner[x | (y << L) | (z << (2 * L))];
            if (o != owner[b]) sets[owner[b]].push_back(o);
        }
    }
    nbr_off.assign(G + 1, 0);
    nbr.clear();
    for (int c = 0; c < G; c++) {
        std::sort(sets[c].begin(), sets[c].end());
        sets[c].erase(std::unique(sets[c].begin(), sets[c].end()), sets[c].end());
        nbr.insert(nbr.end(), sets[c].begin(), sets[c].end());
        nbr_off[c + 1] = (int)nbr.size();
    }
    ctas = G;
    return cudaSuccess;
}

// A run of nsteps >= 2 steps of one pool in one launch: in0 (the output of
// a step) -> buf0 -> buf1 -> buf0 ... and the last step into `last`; maps:
// the face-box tensor maps of in0, buf0 and buf1; ctas, nbr_off, nbr: the
// layout of rd_run_layout (nbr_off, nbr in device memory); flags: ctas *
// kRunFlagStride words of device memory.
template <typename Real>
cudaError_t launch_rd_run_tma(const PoolView<Real> &v, const BlockLists &lists, int ctas, const int *nbr_off,
                              const int *nbr, const Real *H, const unsigned short *meta, double ih2, const Real *in0,
                              Real *buf0, Real *buf1, Real *last, int nsteps, Real rho, double dt, unsigned *nan_flag,
                              unsigned *err_flag, unsigned *flags, const CUtensorMap *maps_in0,
                              const CUtensorMap *maps_buf0, const CUtensorMap *maps_buf1, cudaStream_t s)
{
    if (lists.n_heavy + lists.n_empty <= 0) return cudaSuccess;
    if (nsteps < 2 || nsteps > kMaxRunSteps || !flags || !nbr_off || !nbr) return cudaErrorInvalidValue;
    if (!tma_step_eligible(v) || lists.n_heavy + lists.n_empty != v.nblocks) return cudaErrorInvalidValue;
    PoolSource<Real> src;
    src.heavy = lists.heavy;
    src.empty = lists.empty;
    src.nh = lists.n_heavy;
    src.ne = lists.n_empty;
    src.phi_in = in0;
    src.phi_out = last;
    src.H = H;
    src.pw = v.pw;
    src.pg = v.pg;
    src.meta = meta;
    src.rho = rho;
    src.dt = dt;
    src.L = v.log2_bpd;
    src.nblocks = v.nblocks;
    src.nan_flag = nan_flag;
    StepRun<Real> run;
    run.in0 = in0;
    run.buf[0] = buf0;
    run.buf[1] = buf1;
    run.last = last;
    run.flags = flags;
    run.nbr_off = nbr_off;
    run.nbr = nbr;
    run.nsteps = nsteps;
    TmaMaps<3> m;
    for (int i = 0; i < 3; i++) {
        m.b[0].m[i] = maps_in0[i];
        m.b[1].m[i] = maps_buf0[i];
        m.b[2].m[i] = maps_buf1[i];
    }
    return with_shape<Real>(
        [&](auto sh) { return decltype(sh)::launch_run(src, v.nblocks, ctas, ih2, err_flag, run, m, s); });
}

template <typename Real>
cudaError_t launch_rd_batch_step_tma(const BatchLists &bl, int nactive, int total_items, bool skip_empty,
                                     int log2_bpd, int nblocks, const Real *phi_in, Real *phi_out, const Real *H,
                                     const Real *pw, const Real *pg, const unsigned short *meta, const Real *rho,
                                     const double *dt, double ih2, bool clamped, unsigned *nan_flags,
                                     unsigned *err_flag, const CUtensorMap *maps, int shape, cudaStream_t s)
{
    if (nactive <= 0 || total_items <= 0) return cudaSuccess;
    if (log2_bpd < 0) return cudaErrorInvalidValue;
    BatchSource<Real> src;
    src.hpref = bl.hpref;
    src.epref = bl.epref;
    src.anatomy = bl.anatomy;
    src.hdec = bl.hdec;
    src.edec = bl.edec;
    src.nactive = nactive;
    src.phi_in = phi_in;
    src.phi_out = phi_out;
    src.H = H;
    src.pw = pw;
    src.pg = pg;
    src.meta = meta;
    src.rho = rho;
    src.dt = dt;
    src.L = log2_bpd;
    src.nblocks = nblocks;
    src.nan_flags = nan_flags;
    src.skip_empty = skip_empty;
    return with_shape_code<Real>(shape < 0 ? tma_shape_code() : shape, [&](auto sh) {
        return decltype(sh)::template launch<BatchSource<Real>>(src, total_items, ih2, clamped, err_flag, maps, s);
    });
}

// the shape code a launch with `code` uses (-1: GBFK_TMA_SHAPE, else the
// default of the Real type; a code outside the list: the default)
int tma_shape_effective(int code, int real_bytes)
{
    static const int all[] = {
#define GBFK_TMA_CODE(W, HV, EM) (W * 10 + HV) * 100 + EM,
        GBFK_TMA_SHAPES(GBFK_TMA_CODE)
#undef GBFK_TMA_CODE
    };
    if (code < 0) code = tma_shape_code();
    for (int c : all)
        if (c == code) return code;
    return real_bytes == 4 ? 8208 : 8108;
}

// the launch shapes a batch autotuner may try (codes as for with_shape_code)
int tma_batch_shapes(int *codes, int max_codes)
{
    static const int all[] = {
#define GBFK_TMA_CODE(W, HV, EM) (W * 10 + HV) * 100 + EM,
        GBFK_TMA_SHAPES(GBFK_TMA_CODE)
#undef GBFK_TMA_CODE
    };
    const int n = (int)(sizeof(all) / sizeof(all[0]));
    for (int i = 0; i < n && i < max_codes; i++) codes[i] = all[i];
    return n < max_codes ? n : max_codes;
}

template bool tma_step_eligible<float>(const PoolView<float> &);
template bool tma_step_eligible<double>(const PoolView<double> &);
template cudaError_t launch_rd_step_tma<float>(const PoolView<float> &, const BlockLists &, const float *,
                                               const unsigned short *, double, const float *, bool, float *, float,
                                               double, unsigned *, unsigned *, const CUtensorMap *, bool,
                                               cudaStream_t);
template cudaError_t launch_rd_step_tma<double>(const PoolView<double> &, const BlockLists &, const double *,
                                                const unsigned short *, double, const double *, bool, double *,
                                                double, double, unsigned *, unsigned *, const CUtensorMap *, bool,
                                                cudaStream_t);
template cudaError_t rd_run_layout<float>(const PoolView<float> &, const int *, int, const int *, int, int &,
                                          std::vector<int> &, std::vector<int> &);
template cudaError_t rd_run_layout<double>(const PoolView<double> &, const int *, int, const int *, int, int &,
                                           std::vector<int> &, std::vector<int> &);
template cudaError_t launch_rd_run_tma<float>(const PoolView<float> &, const BlockLists &, int, const int *,
                                              const int *, const float *, const unsigned short *, double,
                                              const float *, float *, float *, float *, int, float, double,
                                              unsigned *, unsigned *, unsigned *, const CUtensorMap *,
                                              const CUtensorMap *, const CUtensorMap *, cudaStream_t);
template cudaError_t launch_rd_run_tma<double>(const PoolView<double> &, const BlockLists &, int, const int *,
                                               const int *, const double *, const unsigned short *, double,
                                               const double *, double *, double *, double *, int, double, double,
                                               unsigned *, unsigned *, unsigned *, const CUtensorMap *,
                                               const CUtensorMap *, const CUtensorMap *, cudaStream_t);
template cudaError_t launch_rd_batch_step_tma<float>(const BatchLists &, int, int, bool, int, int, const float *,
                                                     float *, const float *, const float *, const float *,
                                                     const unsigned short *, const float *, const double *, double,
                                                     bool, unsigned *, unsigned *, const CUtensorMap *, int,
                                                     cudaStream_t);
template cudaError_t launch_rd_batch_step_tma<double>(const BatchLists &, int, int, bool, int, int, const double *,
                                                      double *, const double *, const double *, const double *,
                                                      const unsigned short *, const double *, const double *, double,
                                                      bool, unsigned *, unsigned *, const CUtensorMap *, int,
                                                      cudaStream_t);

}  // namespace gbfk

// The bounded wait of the pipelined step, made to give up: one thread waits
// for the completion of an mbarrier phase that nothing arrives on.  The wait
// ends after its limit and the kernel records that in *err, as the step
// records a copy that never landed, instead of hanging.
namespace gbfk {
__global__ void bounded_wait_probe_kernel(unsigned *err)
{
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        if (!mbar_wait(&bar, 0)) atomicOr(err, 1u);
    }
}
}  // namespace gbfk

extern "C" int gbfk_probe_bounded_wait(int device, double *seconds)
{
    if (cudaSetDevice(device) != cudaSuccess) return GBFK_E_CUDA;
    unsigned *d_err = nullptr, err = 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    float ms = 0;
    cudaError_t e = cudaMalloc(&d_err, sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMemset(d_err, 0, sizeof(unsigned));
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e == cudaSuccess) e = cudaEventRecord(e0, 0);
    if (e == cudaSuccess) {
        gbfk::bounded_wait_probe_kernel<<<1, 32>>>(d_err);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaEventRecord(e1, 0);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (e == cudaSuccess) e = cudaMemcpy(&err, d_err, sizeof(unsigned), cudaMemcpyDeviceToHost);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (d_err) cudaFree(d_err);
    if (e != cudaSuccess) return GBFK_E_CUDA;
    if (seconds) *seconds = ms / 1e3;
    return err ? GBFK_E_TIMEOUT : GBFK_OK;
}
