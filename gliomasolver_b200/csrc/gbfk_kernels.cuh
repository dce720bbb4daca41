// Kernel launchers of the gbfk library (declarations shared by the C ABI).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace gbfk {

constexpr int kBS = 8;
constexpr int kBS3 = 512;
constexpr int kLab = 10;          // lab extent per direction, [-1, 9)
constexpr int kLab3 = 1000;
constexpr int kLabGhosts = 488;
constexpr int kFaceCells = 64;

// Per-topology device data shared by the kernels.
template <typename Real>
struct PoolView {
    const int *slot;       // [nblocks] pool slot of block i
    const int *nbr;        // [nblocks*6] slot of the same-level face neighbour (x-,x+,y-,y+,z-,z+), -1: use ghosts
    const Real *hblk;      // [nblocks] BlockInfo::h[0] in Real
    const Real *gpw;       // [nblocks*488] lab ghosts of p_w (static per topology)
    const Real *gpg;       // [nblocks*488] lab ghosts of p_g
    const Real *gphi;      // [nblocks*488] lab ghosts of phi (refreshed per step where needed)
    const Real *pw;        // pool fields
    const Real *pg;
    int nblocks;
};

template <typename Real>
cudaError_t launch_rd_step(const PoolView<Real> &v, const Real *phi_in, Real *phi_out, Real *dphidt_out,
                           Real Dw, Real Dg, Real rho, double dt, unsigned *nan_flag,
                           cudaStream_t s);

template <typename Real>
cudaError_t launch_fill_ghosts(const int *rows, int64_t nrows, const int64_t *row_ptr, const int *src,
                               const Real *w, const Real *field, Real *ghosts, cudaStream_t s);

template <typename Real>
cudaError_t launch_fwt_details(const PoolView<Real> &v, const Real *phi, double *out, cudaStream_t s);

template <typename Real>
cudaError_t launch_split(const PoolView<Real> &v, int nsplit, const int *parents, const int *children,
                         Real *phi, Real *pw, Real *pg, cudaStream_t s);

template <typename Real>
cudaError_t launch_collapse(int ncollapse, const int *children, const int *parents, Real *phi, Real *pw,
                            Real *pg, cudaStream_t s);

template <typename Real>
cudaError_t launch_dense_scatter(const Real *dense, Real *pool, int n, bool to_pool, cudaStream_t s);

}  // namespace gbfk
