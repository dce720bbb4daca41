// Kernels of the gbfk library: the fused RD step, the ghost fill, the wavelet
// details, split/collapse and the dense <-> block-pool permutation.
#include "gbfk_exact.cuh"
#include "gbfk_kernels.cuh"

namespace gbfk {

// Position of lab cell (x, y, z) in [-1, 9)^3 among a block's 488 ghosts, in
// BlockLab::load's visiting order (MRAG/MRAGcore/MRAGBlockLab.h:256-279);
// -1 for the interior.  Filled by init_ghost_table() at library load.
__constant__ short c_ghost_id[kLab3];

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
// Fused step: ReactionDiffusionOperator<3> + UpdateTumor<3> for one block per
// CTA.  The block and its six face halos of (p_w, p_g, phi) are staged in
// shared memory; the diffusivity df of every staged cell is computed once;
// the harmonic mean of every face is computed once and shared by the two
// cells of the face (it is bit-identical from either side, see
// face_harmonic); then each thread finishes two cells.
template <typename Real>
struct StepSmem {
    Real pw[kLab3], pg[kLab3], ph[kLab3], df[kLab3];
    Real hx[8 * 8 * 9], hy[8 * 8 * 9], hz[8 * 8 * 9];
};

template <typename Real, bool kWriteRhs>
__global__ void __launch_bounds__(256)
rd_step_kernel(PoolView<Real> v, const Real *__restrict__ phi_in, Real *__restrict__ phi_out,
               Real *__restrict__ dphidt_out, Real Dw, Real Dg, Real rho, double dt,
               unsigned *nan_flag)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    StepSmem<Real> &S = *reinterpret_cast<StepSmem<Real> *>(smem_raw);
    const int blk = blockIdx.x;
    const int t = threadIdx.x;
    const int slot = v.slot[blk];
    const int64_t base = (int64_t)slot * kBS3;

    // 1. interior: 512 cells of each field, coalesced
    for (int c = t; c < kBS3; c += 256) {
        const int x = c & 7, y = (c >> 3) & 7, z = c >> 6;
        const int l = lab_index(x, y, z);
        S.pw[l] = v.pw[base + c];
        S.pg[l] = v.pg[base + c];
        S.ph[l] = phi_in[base + c];
    }
    // 2. face halos: same-level neighbours are read directly, the others
    //    from the lab ghosts reconstructed by the ghost fill
    for (int q = t; q < 6 * kFaceCells; q += 256) {
        const int f = q >> 6, p = q & 63;
        int lx, ly, lz, sc;
        face_cell(f, p, lx, ly, lz, sc);
        const int l = lab_index(lx, ly, lz);
        const int nb = v.nbr[blk * 6 + f];
        if (nb >= 0) {
            const int64_t g = (int64_t)nb * kBS3 + sc;
            S.pw[l] = v.pw[g];
            S.pg[l] = v.pg[g];
            S.ph[l] = phi_in[g];
        } else {
            const int64_t g = (int64_t)blk * kLabGhosts + c_ghost_id[l];
            S.pw[l] = v.gpw[g];
            S.pg[l] = v.gpg[g];
            S.ph[l] = v.gphi[g];
        }
    }
    __syncthreads();

    // 3. df = p_w*Dw + p_g*Dg for the interior and the face halos
    for (int c = t; c < kBS3; c += 256) {
        const int l = lab_index(c & 7, (c >> 3) & 7, c >> 6);
        S.df[l] = diffusivity(S.pw[l], S.pg[l], Dw, Dg);
    }
    for (int q = t; q < 6 * kFaceCells; q += 256) {
        int lx, ly, lz, sc;
        face_cell(q >> 6, q & 63, lx, ly, lz, sc);
        const int l = lab_index(lx, ly, lz);
        S.df[l] = diffusivity(S.pw[l], S.pg[l], Dw, Dg);
    }
    __syncthreads();

    // 4. harmonic means of the 3 x 576 faces
    for (int q = t; q < 3 * 576; q += 256) {
        const int d = q / 576, r = q - d * 576;
        const int f = r % 9, a = (r / 9) & 7, b = r / 72;
        int l0, l1;
        Real *H;
        if (d == 0) { l0 = lab_index(f - 1, a, b); l1 = lab_index(f, a, b); H = S.hx; }
        else if (d == 1) { l0 = lab_index(a, f - 1, b); l1 = lab_index(a, f, b); H = S.hy; }
        else { l0 = lab_index(a, b, f - 1); l1 = lab_index(a, b, f); H = S.hz; }
        H[r] = face_harmonic(S.df[l0], S.df[l1]);
    }
    __syncthreads();

    // 5. flux, reaction and update: thread -> (x, y) column, z = t>>6 and +4
    const double h = (double)v.hblk[blk];
    const double ih2 = 1. / (h * h);
    const int x = t & 7, y = (t >> 3) & 7;
    bool bad = false;
#pragma unroll
    for (int k = 0; k < 2; k++) {
        const int z = (t >> 6) + 4 * k;
        const int l = lab_index(x, y, z);
        const Real phi = S.ph[l];
        Real dphidt = (Real)0.;
        if (in_domain(S.pw[l], S.pg[l], phi)) {
            const int ln[6] = {lab_index(x - 1, y, z), lab_index(x + 1, y, z), lab_index(x, y - 1, z),
                               lab_index(x, y + 1, z), lab_index(x, y, z - 1), lab_index(x, y, z + 1)};
            Real chf[6], phn[6];
#pragma unroll
            for (int i = 0; i < 6; i++) {
                phn[i] = S.ph[ln[i]];
                chf[i] = domain_chf(phn[i], S.pw[ln[i]], S.pg[ln[i]]);
            }
            const int rx = (z * 8 + y) * 9, ry = (z * 8 + x) * 9, rz = (y * 8 + x) * 9;
            dphidt = cell_rhs<Real>(S.hx[rx + x], S.hx[rx + x + 1], S.hy[ry + y], S.hy[ry + y + 1],
                                    S.hz[rz + z], S.hz[rz + z + 1], chf, phn, phi, rho, ih2);
        }
        const int c = x + kBS * (y + kBS * z);
        if (kWriteRhs) {
            dphidt_out[base + c] = dphidt;
        } else {
            const Real p = cell_update(phi, dphidt, dt);
            bad |= (p != p);
            phi_out[base + c] = p;
        }
    }
    if (!kWriteRhs && bad) atomicOr(nan_flag, 1u);
}

template <typename Real>
cudaError_t launch_rd_step(const PoolView<Real> &v, const Real *phi_in, Real *phi_out, Real *dphidt_out,
                           Real Dw, Real Dg, Real rho, double dt, unsigned *nan_flag, cudaStream_t s)
{
    if (v.nblocks <= 0) return cudaSuccess;
    const size_t smem = sizeof(StepSmem<Real>);
    if (dphidt_out) {
        auto k = rd_step_kernel<Real, true>;
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k<<<v.nblocks, 256, smem, s>>>(v, phi_in, phi_out, dphidt_out, Dw, Dg, rho, dt, nan_flag);
    } else {
        auto k = rd_step_kernel<Real, false>;
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k<<<v.nblocks, 256, smem, s>>>(v, phi_in, phi_out, dphidt_out, Dw, Dg, rho, dt, nan_flag);
    }
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
    fill_ghosts_kernel<Real><<<(int)nb, 256, 0, s>>>(rows, nrows, row_ptr, src, w, field, ghosts);
    return cudaGetLastError();
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
    const int64_t base = (int64_t)v.slot[blk] * kBS3;
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
    const int64_t base = (int64_t)v.slot[pblk] * kBS3;
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

#define GBFK_INSTANTIATE(Real)                                                                               \
    template cudaError_t launch_rd_step<Real>(const PoolView<Real> &, const Real *, Real *, Real *, Real, Real, \
                                              Real, double, unsigned *, cudaStream_t);                       \
    template cudaError_t launch_fill_ghosts<Real>(const int *, int64_t, const int64_t *, const int *,         \
                                                  const Real *, const Real *, Real *, cudaStream_t);          \
    template cudaError_t launch_fwt_details<Real>(const PoolView<Real> &, const Real *, double *, cudaStream_t); \
    template cudaError_t launch_split<Real>(const PoolView<Real> &, int, const int *, const int *, Real *,     \
                                            Real *, Real *, cudaStream_t);                                    \
    template cudaError_t launch_collapse<Real>(int, const int *, const int *, Real *, Real *, Real *,        \
                                               cudaStream_t);                                                 \
    template cudaError_t launch_dense_scatter<Real>(const Real *, Real *, int, bool, cudaStream_t);

GBFK_INSTANTIATE(float)
GBFK_INSTANTIATE(double)

}  // namespace gbfk
