// Kernels of the gbfk library: the fused RD step, the ghost fill, the wavelet
// details, split/collapse and the dense <-> block-pool permutation.
#include "gbfk_exact.cuh"
#include "gbfk_kernels.cuh"

#include <type_traits>

namespace gbfk {

// Programmatic dependent launch (kernels launched by launch_pdl): wait until
// the previous grid on the stream has completed and its writes are visible,
// then let the next grid be scheduled as this one's CTAs finish.  Without
// the launch attribute both instructions return at once.
__device__ __forceinline__ void pdl_wait_then_release()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <typename K, typename... Args>
cudaError_t launch_pdl(K kernel, int grid, int threads, cudaStream_t s, Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(threads);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}


// Position of lab cell (x, y, z) in [-1, 9)^3 among a block's 488 ghosts, in
// BlockLab::load's visiting order (MRAG/MRAGcore/MRAGBlockLab.h:256-279);
// -1 for the interior.  Filled by init_ghost_table() at library load.
__constant__ short c_ghost_id[kLab3];

// Pool slot of topology block blk.
template <typename Real>
__device__ __forceinline__ int64_t slot_of(const PoolView<Real> &v, int blk)
{
    return v.identity_slots ? (int64_t)blk : (int64_t)v.slot[blk];
}

__host__ __device__ inline int lab_index(int x, int y, int z)
{
    return (x + 1) + kLab * ((y + 1) + kLab * (z + 1));
}

// Lab position and source cell of face cell p (0..63) of face f
// (0: x-, 1: x+, 2: y-, 3: y+, 4: z-, 5: z+).  (a, b) run over the two
// other directions, lower direction fastest.
__device__ __forceinline__ void face_cell(int f, int p, int &lx, int &ly, int &lz, int &src_cell)
{
    const int a = p & 7, b = p >> 3;
    const int d = f >> 1, plus = f & 1;
    const int c_lab = plus ? kBS : -1;      // lab coordinate along d
    const int c_src = plus ? 0 : kBS - 1;   // coordinate inside the neighbour
    if (d == 0) { lx = c_lab; ly = a; lz = b; src_cell = c_src + kBS * (a + kBS * b); }
    else if (d == 1) { lx = a; ly = c_lab; lz = b; src_cell = a + kBS * (c_src + kBS * b); }
    else { lx = a; ly = b; lz = c_lab; src_cell = a + kBS * (b + kBS * c_src); }
}

// ---------------------------------------------------------------------------
// Cell classes: which exact shortcut the step may take for the domain test
// p_w + p_g + phi > 0 (ReactionDiffusionOperator.h:103) and the no-flux test
// chf = phi + p_w + p_g < 0.1 (:115-122, :166-181) of a cell.
//   kEmpty : p_w == 0 and p_g == 0, so chf == phi and the domain test is phi > 0;
//   kTissue: t = p_w + p_g >= 0.1 in Real.  Rounding is monotone, so for
//            phi >= 0 both chf >= t >= 0.1 (no doubling) and t + phi > 0 hold;
//   kOther : evaluated exactly from p_w and p_g.

template <typename Real>
__device__ __forceinline__ unsigned cell_class(Real pw, Real pg)
{
    if (pw == (Real)0 && pg == (Real)0) return kEmpty;
    if (radd(pw, pg) >= (Real)0.1) return kTissue;
    return kOther;
}

// ---------------------------------------------------------------------------
// Static coefficients.  The harmonic means of ReactionDiffusionOperator<3>
// (_harmonic_mean, ReactionDiffusionOperator.h:148-163) depend only on p_w,
// p_g, Dw and Dg, never on phi, so they are computed once per topology and
// coefficient pair instead of on every step.  One CTA per block: the block's
// p_w, p_g and their six face halos are staged in shared memory, df =
// p_w*Dw + p_g*Dg is formed once per staged cell, and the harmonic mean of
// each of the 3 x 576 faces of the block (including its boundary faces, seen
// from this block's own lab) is written to global memory:
//   x faces: H[(z*8 + y)*9 + fx],   fx in [0,9) between x = fx-1 and fx
//   y faces: H[576 + (z*9 + fy)*8 + x]
//   z faces: H[1152 + (fz*8 + y)*8 + x]
// The value is bit-identical from either cell of a face (face_harmonic).
// The same pass writes every cell's 16-bit meta word (indexed like the pool):
//   bits 0-1  the cell's class
//   bits 2-7  neighbour k (x-, x+, y-, y+, z-, z+) is kEmpty
//   bits 8-13 neighbour k is kOther
template <typename Real>
struct FaceSmem {
    Real pw[kLab3], pg[kLab3], df[kLab3];
    unsigned char cl[kLab3];
};

template <typename Real>
__global__ void __launch_bounds__(256)
face_kernel(PoolView<Real> v, Real Dw, Real Dg, Real *__restrict__ H, unsigned short *__restrict__ meta,
            unsigned char *__restrict__ btype)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    FaceSmem<Real> &S = *reinterpret_cast<FaceSmem<Real> *>(smem_raw);
    const int blk = blockIdx.x;
    const int t = threadIdx.x;
    const int64_t base = slot_of(v, blk) * kBS3;
    for (int c = t; c < kBS3; c += 256) {
        const int l = lab_index(c & 7, (c >> 3) & 7, c >> 6);
        S.pw[l] = v.pw[base + c];
        S.pg[l] = v.pg[base + c];
    }
    for (int q = t; q < 6 * kFaceCells; q += 256) {
        const int f = q >> 6, p = q & 63;
        int lx, ly, lz, sc;
        face_cell(f, p, lx, ly, lz, sc);
        const int l = lab_index(lx, ly, lz);
        const int nb = v.nbr[blk * 6 + f];
        if (nb >= 0) {
            S.pw[l] = v.pw[(int64_t)nb * kBS3 + sc];
            S.pg[l] = v.pg[(int64_t)nb * kBS3 + sc];
        } else {
            const int64_t g = (int64_t)blk * kLabGhosts + c_ghost_id[l];
            S.pw[l] = v.gpw[g];
            S.pg[l] = v.gpg[g];
        }
    }
    __syncthreads();
    for (int c = t; c < kBS3; c += 256) {
        const int l = lab_index(c & 7, (c >> 3) & 7, c >> 6);
        S.df[l] = diffusivity(S.pw[l], S.pg[l], Dw, Dg);
        S.cl[l] = (unsigned char)cell_class(S.pw[l], S.pg[l]);
    }
    for (int q = t; q < 6 * kFaceCells; q += 256) {
        int lx, ly, lz, sc;
        face_cell(q >> 6, q & 63, lx, ly, lz, sc);
        const int l = lab_index(lx, ly, lz);
        S.df[l] = diffusivity(S.pw[l], S.pg[l], Dw, Dg);
        S.cl[l] = (unsigned char)cell_class(S.pw[l], S.pg[l]);
    }
    __syncthreads();
    Real *Hb = H + (int64_t)blk * kFacesPerBlock;
    for (int q = t; q < 576; q += 256) {
        {
            const int fx = q % 9, y = (q / 9) & 7, z = q / 72;
            Hb[q] = face_harmonic(S.df[lab_index(fx - 1, y, z)], S.df[lab_index(fx, y, z)]);
        }
        {
            const int x = q & 7, fy = (q >> 3) % 9, z = (q >> 3) / 9;
            Hb[576 + q] = face_harmonic(S.df[lab_index(x, fy - 1, z)], S.df[lab_index(x, fy, z)]);
        }
        {
            const int x = q & 7, y = (q >> 3) & 7, fz = q >> 6;
            Hb[1152 + q] = face_harmonic(S.df[lab_index(x, y, fz - 1)], S.df[lab_index(x, y, fz)]);
        }
    }
    bool all_empty = true, all_tissue = true;
    for (int c = t; c < kBS3; c += 256) {
        const int x = c & 7, y = (c >> 3) & 7, z = c >> 6;
        const int ln[6] = {lab_index(x - 1, y, z), lab_index(x + 1, y, z), lab_index(x, y - 1, z),
                           lab_index(x, y + 1, z), lab_index(x, y, z - 1), lab_index(x, y, z + 1)};
        unsigned m = S.cl[lab_index(x, y, z)];
        for (int k = 0; k < 6; k++) {
            const unsigned ck = S.cl[ln[k]];
            if (ck == kEmpty) m |= 1u << (2 + k);
            if (ck == kOther) m |= 1u << (8 + k);
        }
        meta[base + c] = (unsigned short)m;
        all_empty &= (m == kMetaAllEmpty);
        all_tissue &= (m == kMetaAllTissue);
    }
    all_empty = __syncthreads_and(all_empty);
    all_tissue = __syncthreads_and(all_tissue);
    if (t == 0) btype[blk] = all_empty ? kBlockEmpty : all_tissue ? kBlockTissue : kBlockMixed;
}

template <typename Real>
cudaError_t launch_faces(const PoolView<Real> &v, Real Dw, Real Dg, Real *H, unsigned short *meta,
                         unsigned char *btype, cudaStream_t s)
{
    if (v.nblocks <= 0) return cudaSuccess;
    const size_t smem = sizeof(FaceSmem<Real>);
    auto k = face_kernel<Real>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k<<<v.nblocks, 256, smem, s>>>(v, Dw, Dg, H, meta, btype);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// The step: ReactionDiffusionOperator<3> + UpdateTumor<3> fused, one 8^3
// block per CTA of 128 threads, four consecutive x cells per thread.  phi of
// the block and of its six face halos is staged in shared memory (same-level
// neighbours read directly, coarse-fine faces from the lab ghosts); the
// static face coefficients and meta words come from global memory.  The
// class shortcuts are exact; any other case reads p_w and p_g and evaluates
// the reference expressions.  Cells outside the domain get dphidt = 0, and
// with a finite dt their update phi + dt*0 rounds back to phi, so only the
// clamp remains.
constexpr int kPitch = 16;                  // shared lab row: x in [-1,9) at offsets 3..12
constexpr int kPlane = kPitch * kLab;
constexpr int kStepLab = kPlane * kLab;

__device__ __forceinline__ int lab_p(int x, int y, int z) { return (x + 4) + kPitch * ((y + 1) + kLab * (z + 1)); }

template <typename Real>
__device__ __forceinline__ void lab_pwpg(const PoolView<Real> &v, int blk, int64_t base, int lx, int ly, int lz,
                                         Real &pw, Real &pg)
{
    if (lx >= 0 && lx < kBS && ly >= 0 && ly < kBS && lz >= 0 && lz < kBS) {
        const int64_t g = base + lx + kBS * (ly + kBS * lz);
        pw = v.pw[g];
        pg = v.pg[g];
        return;
    }
    const int f = lx < 0 ? 0 : lx >= kBS ? 1 : ly < 0 ? 2 : ly >= kBS ? 3 : lz < 0 ? 4 : 5;
    const int nb = v.nbr[blk * 6 + f];
    if (nb >= 0) {
        const int sx = (lx + kBS) & 7, sy = (ly + kBS) & 7, sz = (lz + kBS) & 7;
        const int64_t g = (int64_t)nb * kBS3 + sx + kBS * (sy + kBS * sz);
        pw = v.pw[g];
        pg = v.pg[g];
    } else {
        const int64_t g = (int64_t)blk * kLabGhosts + c_ghost_id[lab_index(lx, ly, lz)];
        pw = v.gpw[g];
        pg = v.gpg[g];
    }
}

template <typename Real> struct Vec4;
template <> struct Vec4<float> {
    float v[4];
    __device__ __forceinline__ void load(const float *p)
    {
        const float4 a = __ldg(reinterpret_cast<const float4 *>(p));
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    }
    __device__ __forceinline__ void store(float *p) const
    {
        *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
    }
};
template <> struct Vec4<double> {
    double v[4];
    __device__ __forceinline__ void load(const double *p)
    {
        const double2 a = __ldg(reinterpret_cast<const double2 *>(p));
        const double2 b = __ldg(reinterpret_cast<const double2 *>(p) + 1);
        v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
    }
    __device__ __forceinline__ void store(double *p) const
    {
        reinterpret_cast<double2 *>(p)[0] = make_double2(v[0], v[1]);
        reinterpret_cast<double2 *>(p)[1] = make_double2(v[2], v[3]);
    }
};

// Same-level neighbour block of face f: arithmetic on a uniform periodic
// power-of-two grid, else the neighbour table.
template <typename Real>
__device__ __forceinline__ int face_neighbour(const PoolView<Real> &v, int blk, int f)
{
    if (v.log2_bpd >= 0) {
        const int L = v.log2_bpd, m = (1 << L) - 1;
        int bx = blk & m, by = (blk >> L) & m, bz = blk >> (2 * L);
        const int d = f >> 1, s = (f & 1) ? 1 : -1;
        if (d == 0) bx = (bx + s) & m;
        else if (d == 1) by = (by + s) & m;
        else bz = (bz + s) & m;
        return bx | (by << L) | (bz << (2 * L));
    }
    return v.nbr[blk * 6 + f];
}

// resident CTAs per SM the register allocation targets (FP32 / FP64)
#ifndef GBFK_STEP_MIN_BLOCKS_F32
#define GBFK_STEP_MIN_BLOCKS_F32 16
#endif
#ifndef GBFK_STEP_MIN_BLOCKS_F64
#define GBFK_STEP_MIN_BLOCKS_F64 5
#endif

// The step for one block `blk` (all 128 threads of the CTA call it together;
// it synchronises the CTA).  v.pw/v.pg/v.btype and meta describe the anatomy,
// H the face coefficients of the coefficient pair, phi_in/phi_out the field.
template <typename Real, bool kWriteRhs>
__device__ __forceinline__ void step_block(const PoolView<Real> &v, int blk, Real *__restrict__ ph,
                                           const Real *__restrict__ H, const unsigned short *__restrict__ meta,
                                           const double *__restrict__ ih2blk, const Real *__restrict__ phi_in,
                                           Real *__restrict__ phi_out, Real *__restrict__ dphidt_out, Real rho,
                                           double dt, int dt_finite, unsigned *nan_flag)
{
    const int t = threadIdx.x;
    const int64_t base = slot_of(v, blk) * kBS3;
    const int x4 = (t & 1) * 4, y = (t >> 1) & 7, z = t >> 4;
    const int c0 = x4 + kBS * (y + kBS * z);
    const int l0 = lab_p(x4, y, z);

    // own cells, block type (and meta words if the block is mixed)
    Vec4<Real> p;
    p.load(phi_in + base + c0);
    const unsigned char bt = __ldg(v.btype + blk);
    unsigned mw[4];
    if (bt == kBlockMixed) {
        const uint2 mraw = __ldg(reinterpret_cast<const uint2 *>(meta + base + c0));
        mw[0] = mraw.x & 0xffffu; mw[1] = mraw.x >> 16; mw[2] = mraw.y & 0xffffu; mw[3] = mraw.y >> 16;
    } else {
        const unsigned m = bt == kBlockEmpty ? kMetaAllEmpty : kMetaAllTissue;
        mw[0] = mw[1] = mw[2] = mw[3] = m;
    }
    bool dom[4];
    bool any = false;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const unsigned cls = mw[i] & 3u;
        const Real phi = p.v[i];
        if (cls == kTissue && phi >= (Real)0) dom[i] = true;
        else if (cls == kEmpty) dom[i] = phi > (Real)0;
        else {
            Real pw, pg;
            lab_pwpg(v, blk, base, x4 + i, y, z, pw, pg);
            dom[i] = in_domain(pw, pg, phi);
        }
        any |= dom[i];
    }

    Vec4<Real> out;
    bool bad = false;
    // a block with no cell inside the domain only needs the clamp of the
    // update (dphidt = 0 everywhere): no halo, no face coefficients
    if (!__syncthreads_or(any)) {
#pragma unroll
        for (int i = 0; i < 4; i++) {
            if (kWriteRhs) out.v[i] = (Real)0.;
            else {
                const Real q = dt_finite ? clamp01(p.v[i]) : cell_update(p.v[i], (Real)0., dt);
                bad |= (q != q);
                out.v[i] = q;
            }
        }
        if (kWriteRhs) out.store(dphidt_out + base + c0);
        else out.store(phi_out + base + c0);
        if (!kWriteRhs && bad) atomicOr(nan_flag, 1u);
        return;
    }

    // face halos: 3 per thread, the face index is uniform across a warp
    Real halo[3];
    int hlab[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        const int q = t + 128 * i;
        const int f = q >> 6, pc = q & 63;
        int lx, ly, lz, sc;
        face_cell(f, pc, lx, ly, lz, sc);
        hlab[i] = lab_p(lx, ly, lz);
        const int nb = face_neighbour(v, blk, f);
        if (nb >= 0) halo[i] = phi_in[(int64_t)nb * kBS3 + sc];
        else halo[i] = v.gphi[(int64_t)blk * kLabGhosts + c_ghost_id[lab_index(lx, ly, lz)]];
    }
    // face coefficients of the own cells inside the domain
    Real hx[5];
    Vec4<Real> hym, hyp, hzm, hzp;
    if (any) {
        const Real *Hb = H + (int64_t)blk * kFacesPerBlock;
        const int rx = (z * 8 + y) * 9 + x4;
#pragma unroll
        for (int i = 0; i < 5; i++) hx[i] = __ldg(Hb + rx + i);
        hym.load(Hb + 576 + (z * 9 + y) * 8 + x4);
        hyp.load(Hb + 576 + (z * 9 + y + 1) * 8 + x4);
        hzm.load(Hb + 1152 + (z * 8 + y) * 8 + x4);
        hzp.load(Hb + 1152 + ((z + 1) * 8 + y) * 8 + x4);
    }
    p.store(ph + l0);
#pragma unroll
    for (int i = 0; i < 3; i++) ph[hlab[i]] = halo[i];
    __syncthreads();

    const double ih2 = ih2blk[blk];
    const Real eps = (Real)0.1;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const Real phi = p.v[i];
        Real dphidt = (Real)0.;
        if (dom[i]) {
            const int l = l0 + i;
            Real phn[6];
            phn[0] = i == 0 ? ph[l - 1] : p.v[i - 1];
            phn[1] = i == 3 ? ph[l + 1] : p.v[i + 1];
            phn[2] = ph[l - kPitch];
            phn[3] = ph[l + kPitch];
            phn[4] = ph[l - kPlane];
            phn[5] = ph[l + kPlane];
            bool low[6];
#pragma unroll
            for (int k = 0; k < 6; k++) {
                bool slow;
                if (bt == kBlockTissue) {
                    low[k] = false;
                    slow = !(phn[k] >= (Real)0);
                } else if (bt == kBlockEmpty) {
                    low[k] = phn[k] < eps;
                    slow = false;
                } else if ((mw[i] >> (2 + k)) & 1u) {
                    low[k] = phn[k] < eps;
                    slow = false;
                } else {
                    low[k] = false;
                    slow = ((mw[i] >> (8 + k)) & 1u) || !(phn[k] >= (Real)0);
                }
                if (slow) {
                    const int x = x4 + i;
                    const int nx = x + (k == 0 ? -1 : k == 1 ? 1 : 0);
                    const int ny = y + (k == 2 ? -1 : k == 3 ? 1 : 0);
                    const int nz = z + (k == 4 ? -1 : k == 5 ? 1 : 0);
                    Real pw, pg;
                    lab_pwpg(v, blk, base, nx, ny, nz, pw, pg);
                    low[k] = domain_chf(phn[k], pw, pg) < eps;
                }
            }
            dphidt = cell_rhs_flags<Real>(hx[i], hx[i + 1], hym.v[i], hyp.v[i], hzm.v[i], hzp.v[i], low, phn, phi,
                                          rho, ih2);
        }
        if (kWriteRhs) out.v[i] = dphidt;
        else {
            const Real q = (!dom[i] && dt_finite) ? clamp01(phi) : cell_update(phi, dphidt, dt);
            bad |= (q != q);
            out.v[i] = q;
        }
    }
    if (kWriteRhs) out.store(dphidt_out + base + c0);
    else out.store(phi_out + base + c0);
    if (!kWriteRhs && bad) atomicOr(nan_flag, 1u);
}

template <typename Real, bool kWriteRhs>
__global__ void __launch_bounds__(128, sizeof(Real) == 4 ? GBFK_STEP_MIN_BLOCKS_F32 : GBFK_STEP_MIN_BLOCKS_F64)
rd_step_kernel(PoolView<Real> v, const Real *__restrict__ H, const unsigned short *__restrict__ meta,
               const double *__restrict__ ih2blk, const Real *__restrict__ phi_in, Real *__restrict__ phi_out,
               Real *__restrict__ dphidt_out, Real rho, double dt, int dt_finite, unsigned *nan_flag)
{
    __shared__ __align__(16) Real ph[kStepLab];
    pdl_wait_then_release();
    step_block<Real, kWriteRhs>(v, blockIdx.x, ph, H, meta, ih2blk, phi_in, phi_out, dphidt_out, rho, dt, dt_finite,
                                nan_flag);
}

// Batched step: every sample of the batch has its own phi buffers, face
// coefficients (its own Dw, Dg), rho and dt, and may have its own anatomy.
// blockIdx.x = block, blockIdx.y = group of kSamples consecutive active
// samples; a sample whose horizon is reached (step >= nsteps) is skipped.
template <typename Real, int kSamples>
__global__ void __launch_bounds__(128, sizeof(Real) == 4 ? GBFK_STEP_MIN_BLOCKS_F32 : GBFK_STEP_MIN_BLOCKS_F64)
rd_batch_step_kernel(BatchView<Real> b, int nactive, int step)
{
    __shared__ __align__(16) Real ph[kStepLab];
    const int blk = blockIdx.x;
#pragma unroll 1
    for (int k = 0; k < kSamples; k++) {
        const int s = blockIdx.y * kSamples + k;
        if (s >= nactive) return;
        const SampleView<Real> &sv = b.samples[s];
        if (step >= sv.nsteps) continue;
        PoolView<Real> v = b.pool;
        v.pw = sv.pw;
        v.pg = sv.pg;
        v.btype = sv.btype;
        const int par = step & 1;
        step_block<Real, false>(v, blk, ph, sv.H, sv.meta, b.ih2, par ? sv.phi1 : sv.phi0, par ? sv.phi0 : sv.phi1,
                                nullptr, sv.rho, sv.dt, 1, b.nan_flags + s);
        __syncthreads();
    }
}

template <typename Real>
cudaError_t launch_rd_batch_step(const BatchView<Real> &b, int nactive, int step, int samples_per_cta,
                                 cudaStream_t s)
{
    if (nactive <= 0 || b.pool.nblocks <= 0) return cudaSuccess;
    const int groups = (nactive + samples_per_cta - 1) / samples_per_cta;
    const dim3 grid(b.pool.nblocks, groups);
    switch (samples_per_cta) {
    case 1: rd_batch_step_kernel<Real, 1><<<grid, 128, 0, s>>>(b, nactive, step); break;
    case 2: rd_batch_step_kernel<Real, 2><<<grid, 128, 0, s>>>(b, nactive, step); break;
    case 4: rd_batch_step_kernel<Real, 4><<<grid, 128, 0, s>>>(b, nactive, step); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <typename Real>
cudaError_t launch_rd_step(const PoolView<Real> &v, const Real *H, const unsigned short *meta, const double *ih2,
                           const Real *phi_in, Real *phi_out, Real *dphidt_out, Real rho, double dt,
                           unsigned *nan_flag, cudaStream_t s)
{
    if (v.nblocks <= 0) return cudaSuccess;
    const int dt_finite = isfinite(dt) ? 1 : 0;
    if (dphidt_out)
        return launch_pdl(rd_step_kernel<Real, true>, v.nblocks, 128, s, v, H, meta, ih2, phi_in, phi_out,
                          dphidt_out, rho, dt, dt_finite, nan_flag);
    return launch_pdl(rd_step_kernel<Real, false>, v.nblocks, 128, s, v, H, meta, ih2, phi_in, phi_out, dphidt_out,
                      rho, dt, dt_finite, nan_flag);
}

// ---------------------------------------------------------------------------
// Discrete adjoint of the fused step (uniform grids).  The forward step is
//   pre_i = phi_i + dt * r_i(phi),  phi'_i = clamp(pre_i)
//   r_i   = dom_i * ( ih2 * sum_k H~_ik phi_k - ih2 * (sum_k H~_ik) phi_i + rho phi_i (1 - phi_i) )
// with H~_ik the face coefficient toward neighbour k, doubled by the no-flux
// switch.  The switches (dom, the doubling, the clamp) are piecewise constant
// in phi and are held fixed (their derivative is taken as 0), and rounding is
// treated as exact.  Given lambda' = dL/dphi', one adjoint step forms
//   mu_i     = lambda'_i * [0 < pre_i <= 1]
//   lambda_j = mu_j + dt * ( dom_j mu_j (-ih2 sum_k H~_jk + rho (1 - 2 phi_j))
//                           + ih2 sum_{i nbr j} dom_i mu_i H~_ij )
// and accumulates dL/drho += sum_i mu_i dt dom_i phi_i (1 - phi_i) and
// dL/dDw += sum_i mu_i dt dom_i (diffusive part of r_i) / Dw (the face
// coefficients are homogeneous of degree 1 in (Dw, Dg = 0.1 Dw)).
//
// One launch per adjoint step (adj_fused_kernel): lambda_{k+1} of a block
// needs mu_{k+1} of the block and of its face neighbours, and mu_k of the
// block needs only lambda_{k+1} of the block itself and the forward state
// phi_k.  So the launch for step k first forms lambda_{k+1} in registers
// (phase A, from the mu, cell flags, block status and per-cell "self" term
// of step k + 1 that the previous launch stored), then recomputes the
// forward step of its block exactly like step_block (phase B) and forms
// mu_k, the cell flags (bit 0 = dom, bit 1 + k = coefficient k doubled), the
// block status, the self term of step k and the gradient partials, and
// stores those for the next launch (double-buffered: neighbours still read
// the previous set during this launch).  lambda itself is written only by a
// final launch (lambda_0); the first launch reads lambda_N, the loss
// gradient, instead of phase A.  The self term of a domain cell j is
//   self_j = mu_j * (-ih2 * sum_k H~_jk + rho * (1 - 2 phi_j))
// (0 elsewhere), kept in double, and phase A forms
//   lambda_j = mu_j + dt * ((0 + self_j) + sum_{i nbr j} ih2 H~_ij mu_i).
// A block with no domain cell has mu = lambda' [0 < phi <= 1], no gradient
// or self terms and, unless a face neighbour has a domain cell, lambda = mu.
// The state is block-sparse: mu (and so lambda) vanishes wherever pre = 0,
// i.e. outside the tumour's support.  A block whose lambda_{k+1} is zero (its
// own status says mu_{k+1} = 0 and no face neighbour contributes) gets
// mu_k = 0 without a look at the forward state; a block whose mu is zero
// records kAdjMuZero and writes neither mu, flags nor self terms.  Every
// value equals the dense computation's (a zero block's cells are +0 where
// the dense formulas could produce -0: a sign of zero that no later product
// or sum turns into a different number).

__device__ __forceinline__ void neumaier_add(double &s, double &c, double x)
{
    const double t = s + x;
    if (fabs(s) >= fabs(x)) c += (s - t) + x;
    else c += (x - t) + s;
    s = t;
}

// (s, c) += (xs, xc) for compensated sums: s + xs = t + e exactly (Knuth's
// TwoSum, no branch), the rounding error e joins the compensation terms
__device__ __forceinline__ void two_sum_add(double &s, double &c, double xs, double xc)
{
    const double t = s + xs;
    const double bp = t - s;
    const double e = (s - (t - bp)) + (xs - bp);
    s = t;
    c += xc + e;
}

struct AdjSet {
    void *mu;               // Real per cell (pool order)
    double *self;           // per cell
    unsigned char *flags;   // per cell: bit 0 dom, bit 1 + k coefficient k doubled
    unsigned char *status;  // per block: 0, kAdjDom or kAdjMuZero
};

// Cell mapping of the fused adjoint step: thread t owns the column x = t % 8,
// y = (t / 8) % 8 at z = 4 (t / 64) + i, i = 0..3, so that a warp reads 32
// consecutive cells of a plane from global memory; its lab rows are 24 Reals
// apart (planes 240), which spreads the four rows a warp touches over all 32
// shared-memory banks for every neighbour offset (with 16-Real rows, as the
// one-CTA-per-block kernels use, rows y and y + 2 share banks).
constexpr int kAPitch = 24;
constexpr int kAPlane = kAPitch * kLab;
constexpr int kALab = kAPlane * kLab;

__device__ __forceinline__ int lab_a(int x, int y, int z) { return (x + 1) + kAPitch * (y + 1) + kAPlane * (z + 1); }

// Resident CTAs per SM the fused adjoint step's register allocation targets
// (kCtas).  Measured on a B200 in FP32: 8 CTAs (64 registers, no spills) is
// fastest while the fields stay in L2 (128^3: 0.299 s per config-4 gradient,
// against 0.333 s with 10 and 0.355 s with 12); 12 CTAs (40 registers, a few
// spilled) hide more DRAM latency on larger grids (16 x 256^3: 5.86 s against
// 6.18 s with 8).  FP64 keeps 8.
constexpr int kAdjCtasL2 = 8, kAdjCtasDram = 12;
constexpr int kAdjDramBlocks = 16384;  // grids of at least this many blocks (FP32) use kAdjCtasDram

// Face-halo cell i (0..2) of thread t of the adjoint's 128-thread CTA: cell
// t & 63 of face f = 2 i + (t >> 6) (i = 0: x-, x+; 1: y-, y+; 2: z-, z+),
// the cell face_cell(f, t & 63) gives, with its lab position, its cell in the
// neighbour and the neighbour face_neighbour(v, blk, f) gives.  Written with
// the direction i explicit, which the unrolled loops make a constant.
template <typename Real>
__device__ __forceinline__ void adj_halo(const PoolView<Real> &v, int blk, int i, int t, int &f, int &lab, int &sc,
                                         int &nb)
{
    const int plus = (t >> 6) & 1, a = t & 7, b = (t >> 3) & 7;
    f = 2 * i + plus;
    const int cl = plus ? kBS : -1, cs = plus ? 0 : kBS - 1;
    if (i == 0) {
        lab = lab_a(cl, a, b);
        sc = cs + kBS * (a + kBS * b);
    } else if (i == 1) {
        lab = lab_a(a, cl, b);
        sc = a + kBS * (cs + kBS * b);
    } else {
        lab = lab_a(a, b, cl);
        sc = a + kBS * (b + kBS * cs);
    }
    if (v.log2_bpd >= 0) {  // bx | by << L | bz << 2L, periodic
        const int L = v.log2_bpd, m = (1 << L) - 1, s = plus ? 1 : -1, sh = i * L;
        nb = (blk & ~(m << sh)) | ((((blk >> sh) + s) & m) << sh);
    } else {
        nb = v.nbr[blk * 6 + f];
    }
}

// phi_k of the four cells of thread t and its three face-halo cells
template <typename Real>
__device__ __forceinline__ void adj_load_phi(const PoolView<Real> &v, int blk, const Real *__restrict__ phi,
                                             int64_t base, int c0, int t, Real p[4], Real halo[3])
{
#pragma unroll
    for (int i = 0; i < 4; i++) p[i] = phi[base + c0 + 64 * i];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        int f, lab, sc, nb;
        adj_halo(v, blk, i, t, f, lab, sc, nb);
        halo[i] = phi[(int64_t)nb * kBS3 + sc];
    }
}

__device__ __forceinline__ void cp_async16(void *dst, const void *src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
                 "l"(src)
                 : "memory");
    asm volatile("cp.async.commit_group;" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// kMode: 0 middle, 1 first (lambda_N given), 2 last (write lambda_0); kAbs:
// also sum the magnitudes of the gradient terms (grad_acc slots 4, 5)
template <typename Real, int kMode, bool kAbs, int kCtas>
__global__ void __launch_bounds__(128, kCtas)
adj_fused_kernel(PoolView<Real> v, const Real *__restrict__ H, const unsigned short *__restrict__ meta,
                 const double *__restrict__ ih2blk, const Real *__restrict__ phi, Real *__restrict__ lam,
                 AdjSet prev, AdjSet out, const int *__restrict__ blocks, Real rho, double dt, double inv_Dw,
                 double *__restrict__ grad_acc)
{
    // FP32: the block's face coefficients in shared memory, copied before the
    // wait for the previous launch (they are fixed for the whole run, and so
    // are the block list and 1/h^2); FP64 reads them from global memory
    constexpr bool kHsm = sizeof(Real) == 4;
    __shared__ __align__(16) Real sm[kALab];  // phase A: mu of step k+1; phase B: phi_k
    __shared__ __align__(16) Real sH[kHsm ? kFacesPerBlock : 1];
    __shared__ unsigned char sfl[kALab];
    __shared__ unsigned char sst[8];
    __shared__ double red[kAbs ? 6 : 4][4];
    __shared__ __align__(16) double sacc[kAbs ? 6 : 4];  // this block's gradient slots, prefetched
    const int blk = blocks ? blocks[blockIdx.x] : (int)blockIdx.x, t = threadIdx.x;
    // thread 0 copies the block's gradient slots into shared memory once the
    // launch is known to reach its end (cp.async: no register held, no wait
    // until the slots are updated), so that their load is not the CTA's last
    // round trip; every return after the copy waits for it first
    auto prefetch_acc = [&]() {
        const double *a = grad_acc + (int64_t)blk * kGradSlots;
        cp_async16(sacc, a);
        cp_async16(sacc + 2, a + 2);
        if constexpr (kAbs) cp_async16(sacc + 4, a + 4);
    };
    const double ih2 = ih2blk[blk];
    if constexpr (kHsm) {
        static_assert(kFacesPerBlock % 4 == 0, "float4 copies");
        const float4 *src = reinterpret_cast<const float4 *>(H + (int64_t)blk * kFacesPerBlock);
        for (int q = t; q < kFacesPerBlock / 4; q += blockDim.x) reinterpret_cast<float4 *>(sH)[q] = src[q];
    }
    const int64_t base = slot_of(v, blk) * kBS3;
    const int x = t & 7, y = (t >> 3) & 7, z0 = (t >> 6) * 4;
    const int c0 = x + kBS * (y + kBS * z0);  // cell i is c0 + 64 i
    const int l0 = lab_a(x, y, z0);            // lab cell i is l0 + kAPlane i
    const Real *Hb = kHsm ? sH : H + (int64_t)blk * kFacesPerBlock;
    const int ln[6] = {-1, 1, -kAPitch, kAPitch, -kAPlane, kAPlane};
    // phase B's inputs that no launch writes (block type, meta words) before
    // the wait; after it (kEarlyPhi), phi_k and its face halos, whose loads
    // are then in flight while phase A runs.  Measured on a B200 (config-4
    // gradient at 128^3, FP32): 1.5 % faster; with 12 CTAs per SM the extra
    // live registers spill and 16 x 256^3 was 4 % slower, so that variant
    // loads phi_k in phase B.
    constexpr bool kEarlyPhi = kMode != 2 && sizeof(Real) == 4 && kCtas == kAdjCtasL2;
    const unsigned char bt = v.btype[blk];
    unsigned mw[4];
    if (bt == kBlockMixed) {
#pragma unroll
        for (int i = 0; i < 4; i++) mw[i] = meta[base + c0 + 64 * i];
    } else {
        const unsigned mm = bt == kBlockEmpty ? kMetaAllEmpty : kMetaAllTissue;
        mw[0] = mw[1] = mw[2] = mw[3] = mm;
    }
    pdl_wait_then_release();
    if (kMode == 1 && t == 0) prefetch_acc();
    Real p[4], ph_halo[3];
    if constexpr (kEarlyPhi) adj_load_phi(v, blk, phi, base, c0, t, p, ph_halo);

    // ---- phase A: lambda_{k+1} of this block -------------------------------
    Real lamv[4];
    if (kMode == 1) {
#pragma unroll
        for (int i = 0; i < 4; i++) lamv[i] = lam[base + c0 + 64 * i];
    } else {
        if (t < 7) sst[t] = prev.status[t == 6 ? blk : face_neighbour(v, blk, t)];
        __syncthreads();
        const unsigned self = sst[6];
        bool contrib = false;
#pragma unroll
        for (int f = 0; f < 6; f++) contrib |= sst[f] == kAdjDom;
        if ((self & kAdjMuZero) && !contrib) {
            // lambda_{k+1} = 0 in the block: mu_k = 0 whatever the step does
            if (kMode == 2) {
#pragma unroll
                for (int i = 0; i < 4; i++) lam[base + c0 + 64 * i] = (Real)0;
            } else if (t == 0) {
                out.status[blk] = kAdjMuZero;
            }
            return;
        }
        if (kMode == 0 && t == 0) prefetch_acc();
        const Real *mu_p = (const Real *)prev.mu;
        const bool own = !(self & kAdjMuZero);
        Real m[4];
#pragma unroll
        for (int i = 0; i < 4; i++) m[i] = own ? mu_p[base + c0 + 64 * i] : (Real)0;
        if (!(self & kAdjDom) && !contrib) {
#pragma unroll
            for (int i = 0; i < 4; i++) lamv[i] = m[i];  // no domain cell and no contribution: lambda = mu
        } else {
#pragma unroll
            for (int i = 0; i < 4; i++) {
                sm[l0 + kAPlane * i] = m[i];
                sfl[l0 + kAPlane * i] = own ? prev.flags[base + c0 + 64 * i] : (unsigned char)0;
            }
#pragma unroll
            for (int i = 0; i < 3; i++) {
                int f, l, sc, nb;
                adj_halo(v, blk, i, t, f, l, sc, nb);
                if (sst[f] == kAdjDom) {
                    sm[l] = mu_p[(int64_t)nb * kBS3 + sc];
                    sfl[l] = prev.flags[(int64_t)nb * kBS3 + sc];
                } else {
                    sm[l] = (Real)0;
                    sfl[l] = 0;
                }
            }
            double sf[4];
#pragma unroll
            for (int i = 0; i < 4; i++) sf[i] = (self & kAdjDom) ? prev.self[base + c0 + 64 * i] : 0.;
            __syncthreads();
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const int z = z0 + i, l = l0 + kAPlane * i;
                const int rx = (z * 8 + y) * 9 + x, ry = 576 + (z * 9 + y) * 8 + x, rz = 1152 + (z * 8 + y) * 8 + x;
                const double hf[6] = {(double)Hb[rx], (double)Hb[rx + 1], (double)Hb[ry], (double)Hb[ry + 8],
                                      (double)Hb[rz], (double)Hb[rz + 64]};
                double acc = 0;
                acc += sf[i];
#pragma unroll
                for (int k = 0; k < 6; k++) {
                    // a neighbour outside the domain has mu = +0 (phi <= 0
                    // there, so pre = phi fails 0 < pre), and ih2 H (+0) = +0
                    // leaves acc (never -0: it starts at +0) unchanged, so its
                    // domain bit need not be tested
                    const unsigned fi = sfl[l + ln[k]];
                    const double hik = ((fi >> (1 + (k ^ 1))) & 1u) ? 2. * hf[k] : hf[k];
                    acc += ih2 * hik * (double)sm[l + ln[k]];
                }
                lamv[i] = (Real)((double)m[i] + dt * acc);
            }
            __syncthreads();  // sm and sfl are reused below
        }
        if (kMode == 2) {
#pragma unroll
            for (int i = 0; i < 4; i++) lam[base + c0 + 64 * i] = lamv[i];
            return;
        }
    }

    // ---- phase B: mu_k, cell flags, status and self term of step k --------
    if constexpr (!kEarlyPhi) adj_load_phi(v, blk, phi, base, c0, t, p, ph_halo);
    bool doms[4], any = false;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const Real ph0 = p[i];
        const unsigned cls = mw[i] & 3u;
        if (cls == kTissue && ph0 >= (Real)0) doms[i] = true;
        else if (cls == kEmpty) doms[i] = ph0 > (Real)0;
        else {
            Real pw, pg;
            lab_pwpg(v, blk, base, x, y, z0 + i, pw, pg);
            doms[i] = in_domain(pw, pg, ph0);
        }
        any |= doms[i];
    }
    Real *mu_o = (Real *)out.mu;
    if (!__syncthreads_or(any)) {
        // no cell inside the domain: dphidt = 0, pre = phi, no gradient or self terms
        Real o[4];
        bool nz = false;
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const Real pre = to_real<Real>(__dadd_rn((double)p[i], __dmul_rn(dt, 0.)));
            o[i] = (pre > (Real)0 && pre <= (Real)1) ? lamv[i] : (Real)0;
            nz |= o[i] != (Real)0;
        }
        if (!__syncthreads_or(nz)) {
            if (t == 0) {
                out.status[blk] = kAdjMuZero;
                cp_async_wait_all();
            }
            return;
        }
#pragma unroll
        for (int i = 0; i < 4; i++) {
            mu_o[base + c0 + 64 * i] = o[i];
            out.flags[base + c0 + 64 * i] = 0;
        }
        if (t == 0) {
            out.status[blk] = 0;
            cp_async_wait_all();
        }
        return;
    }
    Real *ph = sm;
#pragma unroll
    for (int i = 0; i < 4; i++) ph[l0 + kAPlane * i] = p[i];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        int f, lab, sc, nb;
        adj_halo(v, blk, i, t, f, lab, sc, nb);
        ph[lab] = ph_halo[i];
    }
    __syncthreads();
    const Real eps = (Real)0.1;
    double grho = 0, grho_c = 0, gdw = 0, gdw_c = 0;
    double arho = 0, adw = 0;  // kAbs
    bool nz = false;
    Real o[4];
    unsigned char fl[4];
    double sfo[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int z = z0 + i;
        const Real ph0 = p[i];
        const bool dom = doms[i];
        unsigned char f = dom ? 1 : 0;
        Real dphidt = (Real)0.;
        double flux_diff = 0, sdf = 0;
        if (dom) {
            const int l = l0 + kAPlane * i;
            Real phn[6];
#pragma unroll
            for (int k = 0; k < 6; k++) phn[k] = ph[l + ln[k]];
            bool low[6];
#pragma unroll
            for (int k = 0; k < 6; k++) {
                bool slow;
                if (bt == kBlockTissue) {  // block-uniform: every neighbour is kTissue
                    low[k] = false;
                    slow = !(phn[k] >= (Real)0);
                } else if ((mw[i] >> (2 + k)) & 1u) {
                    low[k] = phn[k] < eps;
                    slow = false;
                } else {
                    low[k] = false;
                    slow = ((mw[i] >> (8 + k)) & 1u) || !(phn[k] >= (Real)0);
                }
                if (slow) {
                    const int nx = x + (k == 0 ? -1 : k == 1 ? 1 : 0);
                    const int ny = y + (k == 2 ? -1 : k == 3 ? 1 : 0);
                    const int nz2 = z + (k == 4 ? -1 : k == 5 ? 1 : 0);
                    Real pw, pg;
                    lab_pwpg(v, blk, base, nx, ny, nz2, pw, pg);
                    low[k] = domain_chf(phn[k], pw, pg) < eps;
                }
            }
            const int rx = (z * 8 + y) * 9 + x, ry = 576 + (z * 9 + y) * 8 + x, rz = 1152 + (z * 8 + y) * 8 + x;
            Real df[6] = {Hb[rx], Hb[rx + 1], Hb[ry], Hb[ry + 8], Hb[rz], Hb[rz + 64]};
            // _applyNoFluxBC: neighbour k below 0.1 doubles the opposite coefficient k^1
#pragma unroll
            for (int k = 0; k < 6; k++)
                if (low[k]) {
                    df[k ^ 1] = rmul(df[k ^ 1], (Real)2.0);
                    f |= (unsigned char)(1u << (1 + (k ^ 1)));
                }
            Real sin_ = rmul(df[0], phn[0]);
#pragma unroll
            for (int k = 1; k < 6; k++) sin_ = radd(sin_, rmul(df[k], phn[k]));
            const double fluxIn = __dmul_rn(ih2, (double)sin_);
            const Real sdfr = radd(radd(radd(radd(radd(df[0], df[1]), df[2]), df[3]), df[4]), df[5]);
            const double fluxOut = -__dmul_rn((double)rmul(sdfr, ph0), ih2);
            const double reaction = __dmul_rn((double)rmul(rho, ph0), __dadd_rn(1., -(double)ph0));
            dphidt = to_real<Real>(__dadd_rn(__dadd_rn(fluxOut, fluxIn), reaction));
            flux_diff = fluxOut + fluxIn;
#pragma unroll
            for (int k = 0; k < 6; k++) sdf += (double)df[k];
        }
        const Real pre = to_real<Real>(__dadd_rn((double)ph0, __dmul_rn(dt, (double)dphidt)));
        const bool pass = pre > (Real)0 && pre <= (Real)1;
        const Real mv = pass ? lamv[i] : (Real)0;
        o[i] = mv;
        nz |= mv != (Real)0;
        fl[i] = f;
        sfo[i] = dom ? (double)mv * (-ih2 * sdf + (double)rho * (1. - 2. * (double)ph0)) : 0.;
        if (dom && pass) {
            const double tr = (double)mv * dt * (double)ph0 * (1. - (double)ph0);
            const double td = (double)mv * dt * flux_diff * inv_Dw;
            two_sum_add(grho, grho_c, tr, 0.);
            two_sum_add(gdw, gdw_c, td, 0.);
            if (kAbs) {
                arho += fabs(tr);
                adw += fabs(td);
            }
        }
    }
    // a block whose mu is zero everywhere writes neither mu, flags nor self terms
    const bool written = __syncthreads_or(nz);
    if (written) {
#pragma unroll
        for (int i = 0; i < 4; i++) {
            mu_o[base + c0 + 64 * i] = o[i];
            out.flags[base + c0 + 64 * i] = fl[i];
            out.self[base + c0 + 64 * i] = sfo[i];
        }
    }
    if (t == 0) out.status[blk] = written ? kAdjDom : kAdjMuZero;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const double a0 = __shfl_down_sync(0xffffffffu, grho, off), a1 = __shfl_down_sync(0xffffffffu, grho_c, off);
        const double b0 = __shfl_down_sync(0xffffffffu, gdw, off), b1 = __shfl_down_sync(0xffffffffu, gdw_c, off);
        two_sum_add(grho, grho_c, a0, a1);
        two_sum_add(gdw, gdw_c, b0, b1);
        if (kAbs) {
            arho += __shfl_down_sync(0xffffffffu, arho, off);
            adw += __shfl_down_sync(0xffffffffu, adw, off);
        }
    }
    if ((t & 31) == 0) {
        red[0][t >> 5] = grho;
        red[1][t >> 5] = grho_c;
        red[2][t >> 5] = gdw;
        red[3][t >> 5] = gdw_c;
        if constexpr (kAbs) {
            red[4][t >> 5] = arho;
            red[5][t >> 5] = adw;
        }
    }
    __syncthreads();
    if (t == 0) {
        for (int w = 1; w < 4; w++) {
            neumaier_add(red[0][0], red[1][0], red[0][w]);
            neumaier_add(red[0][0], red[1][0], red[1][w]);
            neumaier_add(red[2][0], red[3][0], red[2][w]);
            neumaier_add(red[2][0], red[3][0], red[3][w]);
        }
        cp_async_wait_all();
        double a0 = sacc[0], a1 = sacc[1], a2 = sacc[2], a3 = sacc[3];
        neumaier_add(a0, a1, red[0][0]);
        neumaier_add(a0, a1, red[1][0]);
        neumaier_add(a2, a3, red[2][0]);
        neumaier_add(a2, a3, red[3][0]);
        double *acc = grad_acc + (int64_t)blk * kGradSlots;
        acc[0] = a0;
        acc[1] = a1;
        acc[2] = a2;
        acc[3] = a3;
        if constexpr (kAbs) {
            acc[4] = sacc[4] + (red[4][0] + red[4][1] + red[4][2] + red[4][3]);
            acc[5] = sacc[5] + (red[5][0] + red[5][1] + red[5][2] + red[5][3]);
        }
    }
}

template <typename Real>
cudaError_t launch_adjoint_fused(const PoolView<Real> &v, const Real *H, const unsigned short *meta,
                                 const double *ih2, const Real *phi, Real *lam, const AdjBuffers &prev,
                                 const AdjBuffers &out, int mode, bool abs_terms, const int *blocks, int nlaunch,
                                 Real rho, double dt, double Dw, double *grad_acc, cudaStream_t s)
{
    const int grid = blocks ? nlaunch : v.nblocks;
    if (grid <= 0) return cudaSuccess;
    const AdjSet a = {prev.mu, prev.self, prev.flags, prev.status}, b = {out.mu, out.self, out.flags, out.status};
    auto go = [&](auto kernel) {
        return launch_pdl(kernel, grid, 128, s, v, H, meta, ih2, phi, lam, a, b, blocks, rho, dt, 1. / Dw, grad_acc);
    };
    auto pick = [&](auto ctas) {
        constexpr int C = decltype(ctas)::value;
        if (mode == 1)
            return abs_terms ? go(adj_fused_kernel<Real, 1, true, C>) : go(adj_fused_kernel<Real, 1, false, C>);
        if (mode == 2) return go(adj_fused_kernel<Real, 2, false, C>);  // no step: no gradient terms
        return abs_terms ? go(adj_fused_kernel<Real, 0, true, C>) : go(adj_fused_kernel<Real, 0, false, C>);
    };
    if constexpr (sizeof(Real) == 4)
        if (v.nblocks >= kAdjDramBlocks) return pick(std::integral_constant<int, kAdjCtasDram>());
    return pick(std::integral_constant<int, kAdjCtasL2>());
}

// dL/du of loss = -(L_T1c + L_FLAIR) (HGG_Likelihood.cpp:136-156) on a
// uniform grid, written in pool order; the dump of a uniform grid is the
// identity.  For d = u - uc > 0 the term is constant in u; for d < 0,
// d log(alpha)/du = -2 d/slope and d log(1-alpha)/du = e d/slope / (1 - e/2),
// e = exp(-d^2/slope); at d = 0 both are 0.
__device__ __forceinline__ double bernoulli_dlog(double u, double uc, double is2, bool y)
{
    const double d = u - uc;
    if (!(d < -0.0)) return 0.;
    const double e = exp(-d * d * is2);
    return y ? -2. * d * is2 : e * d * is2 / (1. - 0.5 * e);
}

template <typename Real>
__global__ void loss_grad_kernel(int bpd, const Real *__restrict__ phi, const unsigned char *__restrict__ t1c,
                                 const unsigned char *__restrict__ flair, const int *__restrict__ roi_count,
                                 double t1uc, double t2uc, double is2, Real *__restrict__ lam)
{
    const int n = 8 * bpd;
    const int64_t N = (int64_t)n * n * n;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = i >> 9;
        const int c = (int)(i & 511);
        const int bx = (int)(b % bpd), by = (int)((b / bpd) % bpd), bz = (int)(b / ((int64_t)bpd * bpd));
        const int64_t g = (bx * 8 + (c & 7)) + (int64_t)n * ((by * 8 + ((c >> 3) & 7)) + (int64_t)n * (bz * 8 + (c >> 6)));
        const double u = (double)phi[i];
        // a voxel counts as often as the ROI lists it (every voxel once without a ROI)
        const double w = roi_count ? (double)roi_count[g] : 1.;
        lam[i] = (Real)(-w * (bernoulli_dlog(u, t1uc, is2, t1c[g] != 0) + bernoulli_dlog(u, t2uc, is2, flair[g] != 0)));
    }
}

template <typename Real>
cudaError_t launch_loss_grad(int bpd, const Real *phi, const unsigned char *t1c, const unsigned char *flair,
                             const int *roi_count, double t1uc, double t2uc, double slope, Real *lam, cudaStream_t s)
{
    const int64_t N = (int64_t)512 * bpd * bpd * bpd;
    int64_t nb = (N + 255) / 256;
    if (nb > 148 * 32) nb = 148 * 32;
    loss_grad_kernel<Real><<<(int)nb, 256, 0, s>>>(bpd, phi, t1c, flair, roi_count, t1uc, t2uc, 1. / slope, lam);
    return cudaGetLastError();
}

// How often each voxel of an n^3 grid appears in a list of (x, y, z) points
// (count must be zeroed first).
__global__ void roi_count_kernel(int n, const int *__restrict__ roi, int nroi, int *__restrict__ count)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nroi; k += (int64_t)gridDim.x * blockDim.x)
        atomicAdd(&count[roi[3 * k] + (int64_t)n * (roi[3 * k + 1] + (int64_t)n * roi[3 * k + 2])], 1);
}

cudaError_t launch_roi_count(int n, const int *roi, int nroi, int *count, cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(count, 0, (size_t)n * n * n * sizeof(int), s);
    if (e != cudaSuccess || nroi <= 0) return e;
    int64_t nb = ((int64_t)nroi + 255) / 256;
    if (nb > 148 * 32) nb = 148 * 32;
    roi_count_kernel<<<(int)nb, 256, 0, s>>>(n, roi, nroi, count);
    return cudaGetLastError();
}

// Initial condition c0 = exp(-|x-x0|^2/(2 sigma^2)) where p_w + p_g > 0 (x =
// vertex positions of a uniform bpd^3 grid, pool order), and the reduction
// of dL/dx0 = sum_i lambda0_i c0_i (x_i - x0) / sigma^2 (per CTA partials).
template <typename Real>
__global__ void gaussian_ic_kernel(int bpd, const Real *__restrict__ pw, const Real *__restrict__ pg, double x0,
                                   double y0, double z0, double sigma, Real *__restrict__ out)
{
    const int n = 8 * bpd;
    const int64_t N = (int64_t)n * n * n;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = i >> 9;
        const int c = (int)(i & 511);
        const int bx = (int)(b % bpd), by = (int)((b / bpd) % bpd), bz = (int)(b / ((int64_t)bpd * bpd));
        const double x = (double)(bx * 8 + (c & 7)) / n, y = (double)(by * 8 + ((c >> 3) & 7)) / n,
                     z = (double)(bz * 8 + (c >> 6)) / n;
        const double r2 = (x - x0) * (x - x0) + (y - y0) * (y - y0) + (z - z0) * (z - z0);
        out[i] = (pw[i] + pg[i] > (Real)0) ? (Real)exp(-r2 / (2. * sigma * sigma)) : (Real)0;
    }
}

template <typename Real>
__global__ void __launch_bounds__(256)
x0_grad_kernel(int bpd, const Real *__restrict__ c0, const Real *__restrict__ lam0, double x0, double y0, double z0,
               double sigma, double *__restrict__ partial)
{
    const int n = 8 * bpd;
    const int64_t N = (int64_t)n * n * n;
    double s[3] = {0, 0, 0}, cc[3] = {0, 0, 0};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = i >> 9;
        const int c = (int)(i & 511);
        const int bx = (int)(b % bpd), by = (int)((b / bpd) % bpd), bz = (int)(b / ((int64_t)bpd * bpd));
        const double xs[3] = {(double)(bx * 8 + (c & 7)) / n, (double)(by * 8 + ((c >> 3) & 7)) / n,
                              (double)(bz * 8 + (c >> 6)) / n};
        const double w = (double)lam0[i] * (double)c0[i] / (sigma * sigma);
        neumaier_add(s[0], cc[0], w * (xs[0] - x0));
        neumaier_add(s[1], cc[1], w * (xs[1] - y0));
        neumaier_add(s[2], cc[2], w * (xs[2] - z0));
    }
    __shared__ double red[6][256];
    const int t = threadIdx.x;
    for (int d = 0; d < 3; d++) { red[2 * d][t] = s[d]; red[2 * d + 1][t] = cc[d]; }
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (t < w)
            for (int d = 0; d < 3; d++) {
                neumaier_add(red[2 * d][t], red[2 * d + 1][t], red[2 * d][t + w]);
                neumaier_add(red[2 * d][t], red[2 * d + 1][t], red[2 * d + 1][t + w]);
            }
        __syncthreads();
    }
    if (t < 6) partial[blockIdx.x * 6 + t] = red[t][0];
}

template <typename Real>
cudaError_t launch_gaussian_ic(int bpd, const Real *pw, const Real *pg, const double x0[3], double sigma, Real *out,
                               cudaStream_t s)
{
    const int64_t N = (int64_t)512 * bpd * bpd * bpd;
    int64_t nb = (N + 255) / 256;
    if (nb > 148 * 32) nb = 148 * 32;
    gaussian_ic_kernel<Real><<<(int)nb, 256, 0, s>>>(bpd, pw, pg, x0[0], x0[1], x0[2], sigma, out);
    return cudaGetLastError();
}

template <typename Real>
cudaError_t launch_x0_grad(int bpd, const Real *c0, const Real *lam0, const double x0[3], double sigma,
                           double *partial, int nparts, cudaStream_t s)
{
    x0_grad_kernel<Real><<<nparts, 256, 0, s>>>(bpd, c0, lam0, x0[0], x0[1], x0[2], sigma, partial);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Ghost fill: BlockLab::load step 3 (MRAGBlockLab.h:277-293) for a list of
// rows, ghost = 0; ghost += v * w in Real, entries in list order.
template <typename Real>
__global__ void fill_ghosts_kernel(const int *__restrict__ rows, int64_t nrows,
                                   const int64_t *__restrict__ row_ptr, const int *__restrict__ src,
                                   const Real *__restrict__ w, const Real *__restrict__ field,
                                   Real *__restrict__ ghosts)
{
    pdl_wait_then_release();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nrows;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int r = rows[i];
        Real g = (Real)0;
        for (int64_t k = row_ptr[r]; k < row_ptr[r + 1]; k++) g = radd(g, rmul(field[src[k]], w[k]));
        ghosts[r] = g;
    }
}

template <typename Real>
cudaError_t launch_fill_ghosts(const int *rows, int64_t nrows, const int64_t *row_ptr, const int *src,
                               const Real *w, const Real *field, Real *ghosts, cudaStream_t s)
{
    if (nrows <= 0) return cudaSuccess;
    int64_t nb = (nrows + 255) / 256;
    if (nb > 148 * 32) nb = 148 * 32;
    return launch_pdl(fill_ghosts_kernel<Real>, (int)nb, 256, s, rows, nrows, row_ptr, src, w, field, ghosts);
}

// ---------------------------------------------------------------------------
// Wavelet details (BlockFWT::_fwt, MRAG/MRAGcore/MRAGBlockFWT.h:259-298 with
// _filter :219-257, Interp2ndOrder Ha = {1} on [0,1), Ga = {-.5,1,-.5} on
// [-2,1)): the 448 detail coefficients of a block (64 positions x codes 1..7)
// are computed in parallel, then reduced in the reference's order
// (FWTReport::send then _getDetailMaxMag, :88-120).
template <typename Real>
__device__ Real fwt_filter(const Real *lab, int wx, int wy, int wz, int dx, int dy, int dz)
{
    const Real Ga[3] = {(Real)-0.5, (Real)1., (Real)-0.5};
    const int sx = wx ? -2 : 0, sy = wy ? -2 : 0, sz = wz ? -2 : 0;
    Real result = (Real)0;
    for (int iz = sz; iz < 1; iz++) {
        const Real wZ = wz ? Ga[iz + 2] : (Real)1.;
        for (int iy = sy; iy < 1; iy++) {
            const Real wY = wy ? Ga[iy + 2] : (Real)1.;
            const Real wZwY = rmul(wZ, wY);
            for (int ix = sx; ix < 1; ix++) {
                const Real wX = wx ? Ga[ix + 2] : (Real)1.;
                const Real val = lab[lab_index(2 * dx - ix, 2 * dy - iy, 2 * dz - iz)];
                result = radd(result, rmul(val, rmul(wZwY, wX)));
            }
        }
    }
    return result;
}

template <typename Real>
__global__ void __launch_bounds__(256) fwt_details_kernel(PoolView<Real> v, const Real *__restrict__ phi,
                                                          double *__restrict__ out)
{
    __shared__ Real lab[kLab3];
    __shared__ double det[7][64];
    __shared__ double codemax[7];
    const int blk = blockIdx.x, t = threadIdx.x;
    const int64_t base = slot_of(v, blk) * kBS3;
    for (int c = t; c < kBS3; c += 256) lab[lab_index(c & 7, (c >> 3) & 7, c >> 6)] = phi[base + c];
    // ghosts on the + side only: lab range [0, 9)^3
    for (int q = t; q < 9 * 9 * 9; q += 256) {
        const int x = q % 9, y = (q / 9) % 9, z = q / 81;
        if (x < 8 && y < 8 && z < 8) continue;
        const int l = lab_index(x, y, z);
        lab[l] = v.gphi[(int64_t)blk * kLabGhosts + c_ghost_id[l]];
    }
    __syncthreads();
    for (int q = t; q < 7 * 64; q += 256) {
        const int code = 1 + q / 64, pos = q & 63;
        const int dx = pos & 3, dy = (pos >> 2) & 3, dz = pos >> 4;
        const Real val = fwt_filter(lab, code & 1, (code >> 1) & 1, (code >> 2) & 1, dx, dy, dz);
        det[code - 1][pos] = fabs((double)val);
    }
    __syncthreads();
    if (t < 7) {
        double m = 0.0;  // FWTReport::clear sets the max to 0
        for (int pos = 0; pos < 64; pos++) {
            const double a = det[t][pos];
            m = (a < m) ? m : a;  // std::max(val, maxVal)
        }
        codemax[t] = m;
    }
    __syncthreads();
    if (t == 0) {
        double m = codemax[0];
        for (int c = 1; c < 7; c++) m = (m < codemax[c]) ? codemax[c] : m;
        out[blk] = m;
    }
}

template <typename Real>
cudaError_t launch_fwt_details(const PoolView<Real> &v, const Real *phi, double *out, cudaStream_t s)
{
    if (v.nblocks <= 0) return cudaSuccess;
    fwt_details_kernel<Real><<<v.nblocks, 256, 0, s>>>(v, phi, out);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Split (BlockSplitter::_splitBlocks, MRAGBlockSplitter.h:49-98): fine point d
// of a direction receives Hs(2s-d) * lab(s) from coarse points s in
// {d/2} (d even, weight 1) or {(d-1)/2, (d+1)/2} (d odd, weight .5 each),
// summed in the reference's (sz, sy, sx) order with the weight product in
// double (wZ*wY)*wX rounded to Real.  One CTA per parent; all three fields.
template <typename Real>
__global__ void __launch_bounds__(256) split_kernel(PoolView<Real> v, const int *__restrict__ parents,
                                                    const int *__restrict__ children, Real *phi, Real *pw,
                                                    Real *pg)
{
    __shared__ Real lab[3][kLab3];
    const int i = blockIdx.x, t = threadIdx.x;
    const int pblk = parents[i];
    const int64_t base = slot_of(v, pblk) * kBS3;
    Real *fields[3] = {phi, pw, pg};
    const Real *ghosts[3] = {v.gphi, v.gpw, v.gpg};
    for (int f = 0; f < 3; f++) {
        for (int c = t; c < kBS3; c += 256) lab[f][lab_index(c & 7, (c >> 3) & 7, c >> 6)] = fields[f][base + c];
        for (int q = t; q < 9 * 9 * 9; q += 256) {
            const int x = q % 9, y = (q / 9) % 9, z = q / 81;
            if (x < 8 && y < 8 && z < 8) continue;
            const int l = lab_index(x, y, z);
            lab[f][l] = ghosts[f][(int64_t)pblk * kLabGhosts + c_ghost_id[l]];
        }
    }
    __syncthreads();
    for (int q = t; q < 8 * kBS3; q += 256) {
        const int dx = q & 15, dy = (q >> 4) & 15, dz = q >> 8;   // fine coordinates in [0,16)
        int sxs[2], sys[2], szs[2];
        double wxs[2], wys[2], wzs[2];
        int nx, ny, nz;
        if (dx & 1) { nx = 2; sxs[0] = dx >> 1; sxs[1] = (dx >> 1) + 1; wxs[0] = wxs[1] = 0.5; }
        else { nx = 1; sxs[0] = dx >> 1; wxs[0] = 1.0; }
        if (dy & 1) { ny = 2; sys[0] = dy >> 1; sys[1] = (dy >> 1) + 1; wys[0] = wys[1] = 0.5; }
        else { ny = 1; sys[0] = dy >> 1; wys[0] = 1.0; }
        if (dz & 1) { nz = 2; szs[0] = dz >> 1; szs[1] = (dz >> 1) + 1; wzs[0] = wzs[1] = 0.5; }
        else { nz = 1; szs[0] = dz >> 1; wzs[0] = 1.0; }
        const int cx = dx >> 3, cy = dy >> 3, cz = dz >> 3;
        const int64_t cbase = (int64_t)children[8 * i + cx + 2 * (cy + 2 * cz)] * kBS3;
        const int cc = (dx & 7) + kBS * ((dy & 7) + kBS * (dz & 7));
        for (int f = 0; f < 3; f++) {
            Real acc = (Real)0;
            for (int kz = 0; kz < nz; kz++)
                for (int ky = 0; ky < ny; ky++) {
                    const double wZwY = __dmul_rn(wzs[kz], wys[ky]);
                    for (int kx = 0; kx < nx; kx++) {
                        const Real w = to_real<Real>(__dmul_rn(wZwY, wxs[kx]));
                        acc = radd(acc, rmul(lab[f][lab_index(sxs[kx], sys[ky], szs[kz])], w));
                    }
                }
            fields[f][cbase + cc] = acc;
        }
    }
}

template <typename Real>
cudaError_t launch_split(const PoolView<Real> &v, int nsplit, const int *parents, const int *children,
                         Real *phi, Real *pw, Real *pg, cudaStream_t s)
{
    if (nsplit <= 0) return cudaSuccess;
    split_kernel<Real><<<nsplit, 256, 0, s>>>(v, parents, children, phi, pw, pg);
    return cudaGetLastError();
}

// Collapse (BlockCollapser::_collapseBlocks/_filter, MRAGBlockCollapser.h:
// 22-84): parent = 0 + child(2i) * (1*1*1), the injection of Ha = {1}.
template <typename Real>
__global__ void collapse_kernel(int ncollapse, const int *__restrict__ children, const int *__restrict__ parents,
                                Real *phi, Real *pw, Real *pg)
{
    const int i = blockIdx.x;
    if (i >= ncollapse) return;
    Real *fields[3] = {phi, pw, pg};
    const int64_t pbase = (int64_t)parents[i] * kBS3;
    for (int c = threadIdx.x; c < kBS3; c += blockDim.x) {
        const int X = c & 7, Y = (c >> 3) & 7, Z = c >> 6;
        const int ch = (X >> 2) + 2 * ((Y >> 2) + 2 * (Z >> 2));
        const int64_t cbase = (int64_t)children[8 * i + ch] * kBS3;
        const int sc = 2 * (X & 3) + kBS * (2 * (Y & 3) + kBS * 2 * (Z & 3));
        for (int f = 0; f < 3; f++) fields[f][pbase + c] = radd((Real)0, rmul(fields[f][cbase + sc], (Real)1.));
    }
}

template <typename Real>
cudaError_t launch_collapse(int ncollapse, const int *children, const int *parents, Real *phi, Real *pw,
                            Real *pg, cudaStream_t s)
{
    if (ncollapse <= 0) return cudaSuccess;
    collapse_kernel<Real><<<ncollapse, 256, 0, s>>>(ncollapse, children, parents, phi, pw, pg);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Dense n^3 volume <-> uniform block pool (block (bx,by,bz) in slot
// bx + bpd*(by + bpd*bz)).
template <typename Real>
__global__ void dense_scatter_kernel(const Real *__restrict__ src, Real *__restrict__ dst, int n, bool to_pool)
{
    const int64_t N = (int64_t)n * n * n;
    const int bpd = n / kBS;
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < N; g += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(g % n), y = (int)((g / n) % n), z = (int)(g / ((int64_t)n * n));
        const int64_t slot = (x >> 3) + (int64_t)bpd * ((y >> 3) + (int64_t)bpd * (z >> 3));
        const int64_t p = slot * kBS3 + (x & 7) + kBS * ((y & 7) + kBS * (z & 7));
        if (to_pool) dst[p] = src[g];
        else dst[g] = src[p];
    }
}

// CFL data of the current leaves: the largest local diffusion coefficient
// df_loc = p_w * Dw + p_g * Dg of any cell (formed in Real as
// ReactionDiffusionOperator.h:105 forms it) and the smallest block spacing
// h, reduced by warp shuffles and then across the CTA's warps;
// partial[2c] = max df_loc, partial[2c + 1] = min h of CTA c.  A NaN
// coefficient is skipped (fmax/fmin), like the reference's max, which keeps
// the first argument when a comparison is false.
template <typename Real>
__global__ void __launch_bounds__(256)
cfl_kernel(PoolView<Real> v, Real Dw, Real Dg, double *__restrict__ partial)
{
    __shared__ double sm[2][8];
    double dmax = 0, hmin = INFINITY;
    const int64_t ncells = (int64_t)v.nblocks * kBS3;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < ncells;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int blk = (int)(i >> 9), c = (int)(i & 511);
        const int64_t g = slot_of(v, blk) * kBS3 + c;
        const Real df = radd(rmul(v.pw[g], Dw), rmul(v.pg[g], Dg));
        dmax = fmax(dmax, (double)df);
        if (c == 0) hmin = fmin(hmin, (double)v.hblk[blk]);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        dmax = fmax(dmax, __shfl_down_sync(0xffffffffu, dmax, off));
        hmin = fmin(hmin, __shfl_down_sync(0xffffffffu, hmin, off));
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        sm[0][w] = dmax;
        sm[1][w] = hmin;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < (int)(blockDim.x >> 5); k++) {
            dmax = fmax(dmax, sm[0][k]);
            hmin = fmin(hmin, sm[1][k]);
        }
        partial[2 * blockIdx.x] = dmax;
        partial[2 * blockIdx.x + 1] = hmin;
    }
}

template <typename Real>
cudaError_t launch_cfl(const PoolView<Real> &v, Real Dw, Real Dg, double *partial, int nparts, cudaStream_t s)
{
    if (v.nblocks <= 0 || nparts <= 0) return cudaErrorInvalidValue;
    cfl_kernel<Real><<<nparts, 256, 0, s>>>(v, Dw, Dg, partial);
    return cudaGetLastError();
}

template <typename Real>
cudaError_t launch_dense_scatter(const Real *src, Real *dst, int n, bool to_pool, cudaStream_t s)
{
    const int64_t N = (int64_t)n * n * n;
    int64_t nb = (N + 255) / 256;
    if (nb > 148 * 64) nb = 148 * 64;
    dense_scatter_kernel<Real><<<(int)nb, 256, 0, s>>>(src, dst, n, to_pool);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
void init_ghost_table_host(short *table)
{
    for (int i = 0; i < kLab3; i++) table[i] = -1;
    int k = 0;
    for (int icode = 0; icode < 27; icode++) {
        if (icode == 13) continue;
        const int code[3] = {icode % 3 - 1, (icode / 3) % 3 - 1, (icode / 9) % 3 - 1};
        int s[3], e[3];
        for (int d = 0; d < 3; d++) {
            s[d] = code[d] < 1 ? (code[d] < 0 ? -1 : 0) : kBS;
            e[d] = code[d] < 1 ? (code[d] < 0 ? 0 : kBS) : kBS + 1;
        }
        for (int iz = s[2]; iz < e[2]; iz++)
            for (int iy = s[1]; iy < e[1]; iy++)
                for (int ix = s[0]; ix < e[0]; ix++) table[lab_index(ix, iy, iz)] = (short)k++;
    }
}

cudaError_t upload_ghost_table()
{
    short table[kLab3];
    init_ghost_table_host(table);
    return cudaMemcpyToSymbol(c_ghost_id, table, sizeof(table));
}

// out[b] = 1 when a cell of block b (pool order, identity slots) is > 0
template <typename Real>
__global__ void block_any_positive_kernel(const Real *__restrict__ phi, int nblocks, unsigned char *__restrict__ out)
{
    for (int b = blockIdx.x; b < nblocks; b += gridDim.x) {
        const Real *q = phi + (int64_t)b * kBS3;
        bool any = false;
        for (int c = threadIdx.x; c < kBS3; c += blockDim.x) any |= q[c] > (Real)0;
        any = __syncthreads_or(any);
        if (threadIdx.x == 0) out[b] = any ? 1 : 0;
    }
}

template <typename Real>
cudaError_t launch_block_any_positive(const Real *phi, int nblocks, unsigned char *out, cudaStream_t s)
{
    if (nblocks <= 0) return cudaSuccess;
    block_any_positive_kernel<Real><<<nblocks < 148 * 16 ? nblocks : 148 * 16, 128, 0, s>>>(phi, nblocks, out);
    return cudaGetLastError();
}

#define GBFK_INSTANTIATE(Real)                                                                               \
    template cudaError_t launch_rd_step<Real>(const PoolView<Real> &, const Real *, const unsigned short *,    \
                                              const double *, const Real *, Real *, Real *, Real, double,     \
                                              unsigned *, cudaStream_t);                                      \
    template cudaError_t launch_faces<Real>(const PoolView<Real> &, Real, Real, Real *, unsigned short *,       \
                                            unsigned char *, cudaStream_t);                                   \
    template cudaError_t launch_rd_batch_step<Real>(const BatchView<Real> &, int, int, int, cudaStream_t);      \
    template cudaError_t launch_adjoint_fused<Real>(const PoolView<Real> &, const Real *, const unsigned short *,  \
                                                    const double *, const Real *, Real *, const AdjBuffers &,      \
                                                    const AdjBuffers &, int, bool, const int *, int, Real, double, \
                                                    double, double *, cudaStream_t);                               \
    template cudaError_t launch_block_any_positive<Real>(const Real *, int, unsigned char *, cudaStream_t);      \
    template cudaError_t launch_loss_grad<Real>(int, const Real *, const unsigned char *, const unsigned char *, \
                                                const int *, double, double, double, Real *, cudaStream_t);  \
    template cudaError_t launch_gaussian_ic<Real>(int, const Real *, const Real *, const double *, double, Real *, \
                                                  cudaStream_t);                                             \
    template cudaError_t launch_x0_grad<Real>(int, const Real *, const Real *, const double *, double, double *, \
                                              int, cudaStream_t);                                            \
    template cudaError_t launch_fill_ghosts<Real>(const int *, int64_t, const int64_t *, const int *,         \
                                                  const Real *, const Real *, Real *, cudaStream_t);          \
    template cudaError_t launch_fwt_details<Real>(const PoolView<Real> &, const Real *, double *, cudaStream_t); \
    template cudaError_t launch_split<Real>(const PoolView<Real> &, int, const int *, const int *, Real *,     \
                                            Real *, Real *, cudaStream_t);                                    \
    template cudaError_t launch_collapse<Real>(int, const int *, const int *, Real *, Real *, Real *,        \
                                               cudaStream_t);                                                 \
    template cudaError_t launch_dense_scatter<Real>(const Real *, Real *, int, bool, cudaStream_t); \
    template cudaError_t launch_cfl<Real>(const PoolView<Real> &, Real, Real, double *, int, cudaStream_t);

GBFK_INSTANTIATE(float)
GBFK_INSTANTIATE(double)

}  // namespace gbfk
