// The fused RD step as a persistent, TMA-fed pipeline, for uniform periodic
// power-of-two grids whose blocks sit in pool slots 0..n-1 (the resident
// solve: gbfk_set_uniform).  Results are bit-identical to rd_step_kernel
// (gbfk_kernels.cu), which stays the step of every other topology.
//
// Each CTA owns every G-th block (G CTAs, all resident).  Thread 0 keeps
// kStages blocks in flight; the CTA's k-th block lands in stage k % kStages:
//   - the block's phi (cp.async.bulk, 512 Real);
//   - unless the block is empty (every cell and face-halo cell kEmpty), its
//     six face halos as tensor boxes of the neighbouring blocks
//     (cp.async.bulk.tensor.4d on the pool viewed as [slot][z][y][x]; the
//     x faces as 4-wide boxes so that the inner extent is 16 bytes, the y and
//     z faces as a row set / a plane), and its 1728 face coefficients
//     (cp.async.bulk);
//   - for mixed blocks, its 512 meta words (cp.async.bulk).
// Every copy of a stage completes on the stage's mbarrier.  All waits are
// bounded: a stage that does not complete sets the error word and the CTA
// stops after letting its copies in flight land (also bounded).  The
// threads compute the block from shared memory with the arithmetic of
// step_block and store phi; one CTA barrier per block
// both frees the previous stage for refilling and keeps the timeout
// decision uniform across the CTA.  No load uses cluster multicast.
#include <cuda.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "gbfk_exact.cuh"
#include "gbfk_kernels.cuh"

namespace gbfk {
namespace {

constexpr int kMaxChunk = 4096;  // blocks per CTA (their block-type bytes are staged in shared memory)
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

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
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

// One stage.  Every member starts on a 128-byte boundary (sizes are
// multiples of 128 bytes for float and double).
template <typename Real>
struct alignas(128) Stage {
    Real in[512];           // the block, [z][y][x]
    Real xm[256], xp[256];  // x faces: [z][y][4] boxes of the x- (x = 4..7) / x+ (x = 0..3) neighbour
    Real ym[64], yp[64];    // y faces [z][x]: row y = 7 of the y- / y = 0 of the y+ neighbour
    Real zm[64], zp[64];    // z faces [y][x]: plane z = 7 of the z- / z = 0 of the z+ neighbour
    Real H[kFacesPerBlock];
    unsigned short meta[512];
};
static_assert(sizeof(Stage<float>) % 128 == 0 && sizeof(Stage<double>) % 128 == 0, "stage alignment");

template <typename Real, int kStages>
constexpr size_t stage_smem()
{
    return kStages * sizeof(Stage<Real>) + 256 + kMaxChunk;
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

// p_w, p_g of lab cell (x, y, z) of block blk: the interior or one face halo
template <typename Real>
__device__ __forceinline__ void pwpg_at(const PoolView<Real> &v, int blk, int x, int y, int z, Real &pw, Real &pg)
{
    const int L = v.log2_bpd;
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

// kCells consecutive Real from shared / to global memory in one access
template <typename Real, int N>
__device__ __forceinline__ void vec_lds(const Real *src, Real (&d)[N])
{
    if constexpr (N * sizeof(Real) == 16) {
        const float4 a = *reinterpret_cast<const float4 *>(src);
        memcpy(d, &a, 16);
    } else if constexpr (N * sizeof(Real) == 8) {
        const float2 a = *reinterpret_cast<const float2 *>(src);
        memcpy(d, &a, 8);
    } else {
#pragma unroll
        for (int i = 0; i < N; i++) d[i] = src[i];
    }
}

template <typename Real, int N>
__device__ __forceinline__ void vec_stg(Real *dst, const Real (&d)[N])
{
    if constexpr (N * sizeof(Real) == 16) {
        float4 a;
        memcpy(&a, d, 16);
        *reinterpret_cast<float4 *>(dst) = a;
    } else if constexpr (N * sizeof(Real) == 8) {
        float2 a;
        memcpy(&a, d, 8);
        *reinterpret_cast<float2 *>(dst) = a;
    } else {
#pragma unroll
        for (int i = 0; i < N; i++) dst[i] = d[i];
    }
}

// The no-flux tests of a cell's six neighbours (x-, x+, y-, y+, z-, z+):
// low[k] = chf of neighbour k < 0.1, from its class bits in the meta word
// (kMixed) or, in a tissue block, knowing that every neighbour is kTissue.
template <typename Real, bool kMixed>
__device__ __forceinline__ void neighbour_low(const PoolView<Real> &v, int blk, int x, int y, int z, unsigned mw,
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
            slow = (kMixed && ((mw >> (8 + kk)) & 1u)) || !(phn[kk] >= (Real)0);
        }
        if (slow) {
            const int nx = x + (kk == 0 ? -1 : kk == 1 ? 1 : 0);
            const int ny = y + (kk == 2 ? -1 : kk == 3 ? 1 : 0);
            const int nz = z + (kk == 4 ? -1 : kk == 5 ? 1 : 0);
            Real pw, pg;
            pwpg_at(v, blk, nx, ny, nz, pw, pg);
            low[kk] = domain_chf(phn[kk], pw, pg) < eps;
        }
    }
}

// The cells of one thread in a tissue (kMixed = false) or mixed block: its
// column (x, y) at z = z0 .. z0 + kCells - 1, everything from the stage.
template <typename Real, int kCells, bool kMixed>
__device__ __forceinline__ void column_cells(const PoolView<Real> &v, const Stage<Real> &S, int blk, int x, int y,
                                             int z0, int c0, Real rho, double ih2, double dt, int dt_finite,
                                             Real (&out)[kCells])
{
    Real p[kCells];
    unsigned mw[kCells];
#pragma unroll
    for (int i = 0; i < kCells; i++) {
        p[i] = S.in[c0 + 64 * i];
        mw[i] = kMixed ? (unsigned)S.meta[c0 + 64 * i] : kMetaAllTissue;
    }
#pragma unroll
    for (int i = 0; i < kCells; i++) {
        const Real phi = p[i];
        const int z = z0 + i, c = c0 + 64 * i;
        const unsigned cls = mw[i] & 3u;
        bool dom;
        if (cls == kTissue && phi >= (Real)0) dom = true;
        else if (cls == kEmpty) dom = phi > (Real)0;
        else {
            Real pw, pg;
            pwpg_at(v, blk, x, y, z, pw, pg);
            dom = in_domain(pw, pg, phi);
        }
        if (!dom) {
            out[i] = dt_finite ? clamp01(phi) : cell_update(phi, (Real)0., dt);
            continue;
        }
        // one shared load per neighbour: interior or face halo by address
        Real phn[6];
        phn[0] = *(x > 0 ? &S.in[c - 1] : &S.xm[(z * 8 + y) * 4 + 3]);
        phn[1] = *(x < 7 ? &S.in[c + 1] : &S.xp[(z * 8 + y) * 4]);
        phn[2] = *(y > 0 ? &S.in[c - 8] : &S.ym[z * 8 + x]);
        phn[3] = *(y < 7 ? &S.in[c + 8] : &S.yp[z * 8 + x]);
        phn[4] = i > 0 ? p[i - 1] : *(z > 0 ? &S.in[c - 64] : &S.zm[y * 8 + x]);
        phn[5] = i < kCells - 1 ? p[i + 1] : *(z < 7 ? &S.in[c + 64] : &S.zp[y * 8 + x]);
        bool low[6];
        neighbour_low<Real, kMixed>(v, blk, x, y, z, mw[i], phn, low);
        const int rx = (z * 8 + y) * 9 + x, ry = 576 + (z * 9 + y) * 8 + x, rz = 1152 + (z * 8 + y) * 8 + x;
        const Real dphidt = cell_rhs_flags<Real>(S.H[rx], S.H[rx + 1], S.H[ry], S.H[ry + 8], S.H[rz], S.H[rz + 64],
                                                 low, phn, phi, rho, ih2);
        out[i] = cell_update(phi, dphidt, dt);
    }
}

// A cell of an empty block (every cell and face-halo cell kEmpty) with
// phi > 0: inside the domain, neighbours and coefficients from global memory.
template <typename Real>
__device__ __noinline__ Real empty_cell(const PoolView<Real> &v, int blk, int c, Real phi, const Real *H,
                                        const Real *phi_in, Real rho, double ih2, double dt, int dt_finite)
{
    if (!(phi > (Real)0)) return dt_finite ? clamp01(phi) : cell_update(phi, (Real)0., dt);
    const int L = v.log2_bpd;
    const int x = c & 7, y = (c >> 3) & 7, z = c >> 6;
    const Real *b0 = phi_in + (int64_t)blk * kBS3;
    Real phn[6];
    phn[0] = x > 0 ? b0[c - 1] : phi_in[(int64_t)nb_of(blk, L, 0) * kBS3 + c + 7];
    phn[1] = x < 7 ? b0[c + 1] : phi_in[(int64_t)nb_of(blk, L, 1) * kBS3 + c - 7];
    phn[2] = y > 0 ? b0[c - 8] : phi_in[(int64_t)nb_of(blk, L, 2) * kBS3 + c + 56];
    phn[3] = y < 7 ? b0[c + 8] : phi_in[(int64_t)nb_of(blk, L, 3) * kBS3 + c - 56];
    phn[4] = z > 0 ? b0[c - 64] : phi_in[(int64_t)nb_of(blk, L, 4) * kBS3 + c + 448];
    phn[5] = z < 7 ? b0[c + 64] : phi_in[(int64_t)nb_of(blk, L, 5) * kBS3 + c - 448];
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

// CTA c of G handles blocks c, c + G, c + 2G, ... (interleaved, so that the
// tissue blocks of the anatomy spread evenly over the CTAs).  Warp kWarps is
// the producer: its lane 0 refills a stage once every consumer warp has
// released it (the stage's `empty` barrier) and puts the next block in
// flight (its `full` barrier).  The kWarps consumer warps never wait for one
// another: consumer thread t owns the column x = t % 8, y = (t / 8) % 8 and
// kCells consecutive z from (t / 64) * kCells of every block, waits for the
// block's stage, computes and stores its cells and releases the stage.  A
// warp reads 32 consecutive cells of a z plane from shared memory (no bank
// conflicts) and stores 32 consecutive cells.
template <typename Real, int kWarps, int kStages>
__global__ void __launch_bounds__((kWarps + 1) * 32)
rd_step_tma_kernel(PoolView<Real> v, const Real *__restrict__ H, const unsigned short *__restrict__ meta, double ih2,
                   const Real *__restrict__ phi_in, Real *__restrict__ phi_out, Real rho, double dt, int dt_finite,
                   unsigned *nan_flag, unsigned *err_flag, const __grid_constant__ CUtensorMap map_x,
                   const __grid_constant__ CUtensorMap map_y, const __grid_constant__ CUtensorMap map_z)
{
    constexpr int kThreads = kWarps * 32;  // consumer threads
    constexpr int kCells = kBS3 / kThreads;
    static_assert(kCells * kThreads == kBS3 && kCells >= 1 && kCells <= 8, "consumer warps per block");
    extern __shared__ __align__(128) unsigned char smem[];
    Stage<Real> *st = reinterpret_cast<Stage<Real> *>(smem);
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + kStages * sizeof(Stage<Real>));
    uint64_t *empty = full + kStages;
    unsigned char *sbt = smem + kStages * sizeof(Stage<Real>) + 256;
    const int t = threadIdx.x;
    const int G = gridDim.x;
    const int nmine = v.nblocks > (int)blockIdx.x ? (v.nblocks - 1 - (int)blockIdx.x) / G + 1 : 0;
    if (nmine <= 0) return;  // uniform across the CTA
    for (int i = t; i < nmine; i += blockDim.x) sbt[i] = v.btype[blockIdx.x + i * G];
    if (t == 0) {
        for (int s = 0; s < kStages; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], kWarps);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();  // the only CTA-wide barrier

    const int L = v.log2_bpd;
    if (t >= kThreads) {
        // producer warp
        if (t != kThreads) return;
        int issued = 0;
        for (; issued < nmine; issued++) {
            const int k = issued, s = k % kStages;
            if (k >= kStages && !mbar_wait(&empty[s], ((k / kStages) - 1) & 1)) {
                atomicOr(err_flag, 1u);
                break;
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            const int blk = blockIdx.x + k * G;
            Stage<Real> &S = st[s];
            uint64_t *bar = &full[s];
            const unsigned char bt = sbt[k];
            uint32_t bytes = 512 * sizeof(Real);
            if (bt != kBlockEmpty) bytes += (2 * 256 + 4 * 64 + kFacesPerBlock) * sizeof(Real);
            if (bt == kBlockMixed) bytes += 512 * sizeof(unsigned short);
            mbar_arrive_expect_tx(bar, bytes);
            bulk_g2s(S.in, phi_in + (int64_t)blk * kBS3, 512 * sizeof(Real), bar);
            if (bt != kBlockEmpty) {
                box_g2s(S.xm, &map_x, 4, 0, 0, nb_of(blk, L, 0), bar);
                box_g2s(S.xp, &map_x, 0, 0, 0, nb_of(blk, L, 1), bar);
                box_g2s(S.ym, &map_y, 0, 7, 0, nb_of(blk, L, 2), bar);
                box_g2s(S.yp, &map_y, 0, 0, 0, nb_of(blk, L, 3), bar);
                box_g2s(S.zm, &map_z, 0, 0, 7, nb_of(blk, L, 4), bar);
                box_g2s(S.zp, &map_z, 0, 0, 0, nb_of(blk, L, 5), bar);
                bulk_g2s(S.H, H + (int64_t)blk * kFacesPerBlock, kFacesPerBlock * sizeof(Real), bar);
            }
            if (bt == kBlockMixed) bulk_g2s(S.meta, meta + (int64_t)blk * kBS3, 512 * sizeof(unsigned short), bar);
        }
        // the CTA's shared memory must outlive every copy in flight (bounded)
        for (int j = issued - kStages > 0 ? issued - kStages : 0; j < issued; j++)
            mbar_wait(&full[j % kStages], (j / kStages) & 1);
        return;
    }

    const int lane = t & 31;
    const int x = t & 7, y = (t >> 3) & 7, z0 = (t >> 6) * kCells;
    const int c0 = x + kBS * (y + kBS * z0);
    const int ce = t * kCells;  // empty blocks: kCells consecutive cells
    bool bad = false;
    for (int k = 0; k < nmine; k++) {
        const int s = k % kStages;
        if (!__all_sync(0xffffffffu, mbar_wait(&full[s], (k / kStages) & 1))) {
            if (lane == 0) atomicOr(err_flag, 1u);
            break;
        }
        const Stage<Real> &S = st[s];
        const int blk = blockIdx.x + k * G;
        const unsigned char bt = sbt[k];
        Real *ob = phi_out + (int64_t)blk * kBS3;
        if (bt == kBlockEmpty) {
            Real p[kCells], out[kCells];
            vec_lds<Real, kCells>(S.in + ce, p);
            bool any = false;
#pragma unroll
            for (int i = 0; i < kCells; i++) any |= p[i] > (Real)0;  // the domain test of a kEmpty cell
            if (!any) {
#pragma unroll
                for (int i = 0; i < kCells; i++)
                    out[i] = dt_finite ? clamp01(p[i]) : cell_update(p[i], (Real)0., dt);
            } else {
                // tumour outside the anatomy: the stage holds no halo or
                // coefficients of an empty block, read them from global memory
#pragma unroll
                for (int i = 0; i < kCells; i++)
                    out[i] = empty_cell(v, blk, ce + i, p[i], H, phi_in, rho, ih2, dt, dt_finite);
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[s]);
#pragma unroll
            for (int i = 0; i < kCells; i++) bad |= (out[i] != out[i]);
            vec_stg<Real, kCells>(ob + ce, out);
            continue;
        }
        Real out[kCells];
        if (bt == kBlockTissue)
            column_cells<Real, kCells, false>(v, S, blk, x, y, z0, c0, rho, ih2, dt, dt_finite, out);
        else
            column_cells<Real, kCells, true>(v, S, blk, x, y, z0, c0, rho, ih2, dt, dt_finite, out);
        // every shared read of this warp is done: release the stage
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
#pragma unroll
        for (int i = 0; i < kCells; i++) {
            bad |= (out[i] != out[i]);
            ob[c0 + 64 * i] = out[i];
        }
    }
    if (bad) atomicOr(nan_flag, 1u);
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

// Whether the pipelined step applies to a view: uniform periodic 2^L grid,
// identity slots, and per-CTA block counts that fit the kernel's block-type
// buffer.
template <typename Real>
bool tma_step_eligible(const PoolView<Real> &v)
{
    return v.log2_bpd >= 0 && v.identity_slots && v.nblocks > 0 && v.nblocks <= 148 * kMaxChunk;
}

namespace {

// One launch shape: consumer warps per CTA and stages in flight, with its grid
// (resident CTAs on this part) taken once per process.
template <typename Real, int kWarps, int kStages>
cudaError_t launch_shape(const PoolView<Real> &v, const Real *H, const unsigned short *meta, double ih2,
                         const Real *phi_in, Real *phi_out, Real rho, double dt, unsigned *nan_flag,
                         unsigned *err_flag, const CUtensorMap *maps, cudaStream_t s)
{
    static int grid = 0;
    static std::mutex mu;
    constexpr int kThreads = (kWarps + 1) * 32;
    auto k = rd_step_tma_kernel<Real, kWarps, kStages>;
    constexpr size_t smem = stage_smem<Real, kStages>();
    {
        std::lock_guard<std::mutex> lk(mu);
        if (!grid) {
            cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
            int dev = 0, sms = 0, per_sm = 0;
            if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
            if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
            if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kThreads, smem)) != cudaSuccess)
                return e;
            grid = sms * (per_sm > 0 ? per_sm : 1);
        }
    }
    const int nctas = v.nblocks < grid ? v.nblocks : grid;
    if ((v.nblocks + nctas - 1) / nctas > kMaxChunk) return cudaErrorInvalidValue;
    k<<<nctas, kThreads, smem, s>>>(v, H, meta, ih2, phi_in, phi_out, rho, dt, isfinite(dt) ? 1 : 0, nan_flag,
                                     err_flag, maps[0], maps[1], maps[2]);
    return cudaGetLastError();
}

// launch shape from GBFK_TMA_SHAPE="consumer warps,stages" (a tuning knob), else the default
int tma_shape_code()
{
    static int code = -1;
    static std::once_flag once;
    std::call_once(once, [] {
        code = 8 * 10 + 4;
        if (const char *e = getenv("GBFK_TMA_SHAPE")) {
            int th = 0, stg = 0;
            if (sscanf(e, "%d,%d", &th, &stg) == 2) code = th * 10 + stg;
        }
    });
    return code;
}

}  // namespace

template <typename Real>
cudaError_t launch_rd_step_tma(const PoolView<Real> &v, const Real *H, const unsigned short *meta, double ih2,
                               const Real *phi_in, Real *phi_out, Real rho, double dt, unsigned *nan_flag,
                               unsigned *err_flag, const CUtensorMap *maps, cudaStream_t s)
{
    if (v.nblocks <= 0) return cudaSuccess;
    if (!tma_step_eligible(v)) return cudaErrorInvalidValue;
#define GBFK_TMA_SHAPE(TH, ST)                                                                                   \
    case TH * 10 + ST:                                                                                           \
        return launch_shape<Real, TH, ST>(v, H, meta, ih2, phi_in, phi_out, rho, dt, nan_flag, err_flag, maps, s);
    switch (tma_shape_code()) {
        GBFK_TMA_SHAPE(4, 2)
        GBFK_TMA_SHAPE(4, 3)
        GBFK_TMA_SHAPE(4, 4)
        GBFK_TMA_SHAPE(8, 2)
        GBFK_TMA_SHAPE(8, 3)
        GBFK_TMA_SHAPE(8, 6)
        GBFK_TMA_SHAPE(16, 2)
        GBFK_TMA_SHAPE(16, 3)
        GBFK_TMA_SHAPE(16, 4)
    default:
        return launch_shape<Real, 8, 4>(v, H, meta, ih2, phi_in, phi_out, rho, dt, nan_flag, err_flag, maps, s);
    }
#undef GBFK_TMA_SHAPE
}

template bool tma_step_eligible<float>(const PoolView<float> &);
template bool tma_step_eligible<double>(const PoolView<double> &);
template cudaError_t launch_rd_step_tma<float>(const PoolView<float> &, const float *, const unsigned short *, double,
                                               const float *, float *, float, double, unsigned *, unsigned *,
                                               const CUtensorMap *, cudaStream_t);
template cudaError_t launch_rd_step_tma<double>(const PoolView<double> &, const double *, const unsigned short *,
                                                double, const double *, double *, double, double, unsigned *,
                                                unsigned *, const CUtensorMap *, cudaStream_t);

}  // namespace gbfk
