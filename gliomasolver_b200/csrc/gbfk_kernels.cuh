// Kernel launchers of the gbfk library (declarations shared by the C ABI).
#pragma once

#include <vector>
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

namespace gbfk {

constexpr int kBS = 8;
constexpr int kBS3 = 512;
constexpr int kLab = 10;          // lab extent per direction, [-1, 9)
constexpr int kLab3 = 1000;
constexpr int kLabGhosts = 488;
constexpr int kFaceCells = 64;
constexpr int kFacesPerBlock = 3 * 576;  // x, y, z faces of a block incl. its boundary faces
constexpr int kGradSlots = 6;            // adjoint gradient partials per block: rho (sum, comp), Dw (sum, comp),
                                         // and the sums of the magnitudes of their terms (rho, Dw)

// cell classes for the step's exact shortcuts (see cell_class)
constexpr unsigned char kEmpty = 0, kTissue = 1, kOther = 2;

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
    const unsigned char *btype;  // [nblocks] block type of the step (kBlockEmpty / kBlockTissue / kBlockMixed)
    int nblocks;
    int identity_slots;    // slot[i] == i for every block
    int log2_bpd;          // uniform periodic grid of 2^log2_bpd blocks per direction, else -1
};

// Block types: every cell of the block and of its face halos is kEmpty
// (kBlockEmpty) or kTissue (kBlockTissue); otherwise the per-cell meta words
// are read (kBlockMixed).
constexpr unsigned char kBlockEmpty = 0, kBlockTissue = 1, kBlockMixed = 2;
// meta words of a cell whose own class and all six neighbour classes are kEmpty / kTissue
constexpr unsigned kMetaAllEmpty = kEmpty | (0x3fu << 2);
constexpr unsigned kMetaAllTissue = kTissue;

// One sample of a batch (device pointers).
template <typename Real>
struct SampleView {
    const Real *pw, *pg;           // anatomy (pool order)
    const unsigned char *btype;    // block types of that anatomy
    const unsigned short *meta;    // meta words of that anatomy
    const Real *H;                 // face coefficients of (anatomy, Dw, Dg)
    Real *phi0, *phi1;             // ping-pong fields; step k reads phi[k & 1]
    Real rho;
    double dt;
    int nsteps;
};

// A batch: one uniform topology, per-sample views (sorted by horizon,
// longest first, so the active samples of a step are a prefix).
template <typename Real>
struct BatchView {
    PoolView<Real> pool;           // topology (slot/nbr/log2_bpd/identity) shared by the samples
    const SampleView<Real> *samples;
    const double *ih2;
    unsigned *nan_flags;           // one per sample
};

template <typename Real>
cudaError_t launch_rd_batch_step(const BatchView<Real> &b, int nactive, int step, int samples_per_cta,
                                 cudaStream_t s);

// Harmonic means of all faces of every block for (Dw, Dg): H[nblocks * 1728],
// and the per-cell meta words (class + neighbour class masks, pool-indexed).
template <typename Real>
cudaError_t launch_faces(const PoolView<Real> &v, Real Dw, Real Dg, Real *H, unsigned short *meta,
                         unsigned char *btype, cudaStream_t s);

// One fused step (or, with dphidt_out, the operator alone).
template <typename Real>
cudaError_t launch_rd_step(const PoolView<Real> &v, const Real *H, const unsigned short *meta, const double *ih2,
                           const Real *phi_in, Real *phi_out, Real *dphidt_out, Real rho, double dt,
                           unsigned *nan_flag, cudaStream_t s);

// The same step as a persistent TMA-fed pipeline (gbfk_step_tma.cu): uniform
// periodic power-of-two grids with identity slots only (tma_step_eligible).
// lists: the blocks that need halos and face coefficients (heavy: entries
// block * 4 + block type, mixed blocks first) and the empty ones (entries:
// block), together every block once; maps: the three face-box tensor maps of
// phi_in (make_pool_tensor_maps); ih2: the grid's 1/(h*h); clamped: phi_in
// is the output of a step (every value +0 <= phi <= 1 or NaN), which lets
// the kernel skip the negativity tests; err_flag: set when a wait of the
// pipeline timed out; skip_empty: the empty blocks of phi_in and phi_out
// already hold +0 (and the step would keep it: dt finite), so only the heavy
// blocks run.
struct BlockLists {
    const int *heavy;
    int n_heavy;
    const int *empty;
    int n_empty;
};
template <typename Real>
bool tma_step_eligible(const PoolView<Real> &v);
template <typename Real>
cudaError_t launch_rd_step_tma(const PoolView<Real> &v, const BlockLists &lists, const Real *H,
                               const unsigned short *meta, double ih2, const Real *phi_in, bool clamped,
                               Real *phi_out, Real rho, double dt, unsigned *nan_flag, unsigned *err_flag,
                               const CUtensorMap *maps, bool skip_empty, cudaStream_t s);
cudaError_t make_pool_tensor_maps(void *base, int nslots, int real_bytes, CUtensorMap maps[3]);
// A run of nsteps (2 .. kMaxRunSteps) steps of the pipelined step in one
// cooperative launch: in0 (the output of a step) -> buf0 -> buf1 -> buf0 ...,
// the last step into `last`; the results are those of nsteps launches.  Each
// CTA keeps its blocks for the whole run and, between steps, waits only for
// the CTAs that own face neighbours of its blocks (a step flag per CTA,
// kRunFlagStride words apart; rd_run_layout gives the CTA count and the
// neighbour lists, which the launch takes in device memory).  maps_*: the
// face-box tensor maps of in0, buf0, buf1.  The error word of the pipelined
// steps: bit 0 a copy or slot wait gave up (after about a second), bit 1 a
// CTA's work list overflowed; the wait that gave up: bit 3 a consumer's
// heavy slot, 4 its empty slot, 5 the producer's free heavy slot, 6 its
// free empty slot, 7 a step boundary (this CTA's or a neighbour's), 8 the
// wait for every consumer warp's stores.
constexpr int kMaxRunSteps = 1 << 20;
constexpr int kRunFlagStride = 32;
template <typename Real>
cudaError_t rd_run_layout(const PoolView<Real> &v, const int *heavy, int n_heavy, const int *empty, int n_empty,
                          int &ctas, std::vector<int> &nbr_off, std::vector<int> &nbr);
template <typename Real>
cudaError_t launch_rd_run_tma(const PoolView<Real> &v, const BlockLists &lists, int ctas, const int *nbr_off,
                              const int *nbr, const Real *H, const unsigned short *meta, double ih2, const Real *in0,
                              Real *buf0, Real *buf1, Real *last, int nsteps, Real rho, double dt, unsigned *nan_flag,
                              unsigned *err_flag, unsigned *flags, const CUtensorMap *maps_in0,
                              const CUtensorMap *maps_buf0, const CUtensorMap *maps_buf1, cudaStream_t s);

// The same for a step of a TMCMC batch: every active sample (positions
// 0 .. nactive-1) of one uniform 2^log2_bpd grid.  Per-position fields are
// consecutive pools of nblocks blocks (phi_in/phi_out, H); per-anatomy ones
// too (pw, pg, meta).  bl: per-anatomy heavy/empty block lists and the
// prefix sums of their lengths over the positions; total_items = blocks of
// all active samples; rho, dt, nan_flags per position; maps: the face-box
// tensor maps of the phi_in buffer (all positions).  skip_empty: the empty
// blocks of every active sample already hold their output in phi_out (and
// phi_in); total_items then counts the heavy blocks only.
struct BatchLists {
    const int *lists;     // per anatomy: heavy entries (block * 4 + type), then empty entries (block)
    const int *list_off;  // [2a]: offset of anatomy a's heavy entries, [2a + 1]: of its empty entries
    const int *hpref;     // [positions + 1]: heavy blocks of positions before p
    const int *epref;     // [positions + 1]: empty blocks of positions before p
    const int *anatomy;   // [positions]
    // the items decoded once per run: heavy item g is (position, block * 4 +
    // type) = hdec[g], empty item g is (position, block * 4) = edec[g]
    const int2 *hdec, *edec;
};
template <typename Real>
cudaError_t launch_rd_batch_step_tma(const BatchLists &bl, int nactive, int total_items, bool skip_empty,
                                     int log2_bpd, int nblocks, const Real *phi_in, Real *phi_out, const Real *H,
                                     const Real *pw, const Real *pg, const unsigned short *meta, const Real *rho,
                                     const double *dt, double ih2, bool clamped, unsigned *nan_flags,
                                     unsigned *err_flag, const CUtensorMap *maps, int shape, cudaStream_t s);
// launch shapes of the pipelined step a batch may use: codes
// consumer warps * 1000 + heavy slots * 100 + empty slots (shape -1 above:
// the default, or GBFK_TMA_SHAPE); returns how many were written
int tma_batch_shapes(int *codes, int max_codes);
int tma_shape_effective(int code, int real_bytes);

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

// Finest-uniform dump of phi (double, gpd^3, zeroed first).
template <typename Real>
cudaError_t launch_uq_dump(const int *slot, const Real *origin, const Real *hblk, int nblocks, const Real *phi,
                           int gpd, double *out, cudaStream_t s);

struct LikelihoodParams {
    double pet_sigma2, pet_scale, t1_uc, t2_uc, slope;
    int step_pet, step_mri;
};

// out[0..3] = L_PET, L_T1c, L_FLAIR, their sum; partial holds nparts * 7 doubles.
cudaError_t launch_likelihood(const double *model, int n, const unsigned char *t1c, const unsigned char *flair,
                              const double *pet, const int *roi, int nroi, const LikelihoodParams &p,
                              double *partial, int nparts, double *out, cudaStream_t s);

// Discrete adjoint (uniform grids): one adjoint step per launch
// (adj_fused_kernel).  The state of an adjoint step kept between launches,
// double-buffered: per cell mu (Real), the self term (double) and the switch
// flags, per block the status.  mode 1: the first step, lambda' from lam
// (the loss gradient); mode 0: lambda' from prev; mode 2: no step, lambda
// from prev written to lam (lambda_0).  blocks: NULL (one CTA per block) or
// the nlaunch blocks to run, one CTA each; every other block must hold
// status kAdjMuZero in both sets and contribute nothing to the listed ones'
// lambda (the caller's list: every block that can hold a domain cell, and
// their face neighbours).  grad_acc: nblocks * kGradSlots
// doubles (rho sum/comp, Dw sum/comp, and with abs_terms the sums of the
// terms' magnitudes for rho and Dw), accumulated per block.
constexpr int kAdjFlagBytesPerBlock = kBS3 + 1;  // cell flags, then the block's status
// Per-block status of an adjoint step: exactly one of 0 (mu not zero, no
// domain cell), kAdjDom (mu not zero, a domain cell) and kAdjMuZero (mu is
// zero in every cell; its mu values, cell flags and self terms are not
// written, and the block contributes nothing to any lambda).
constexpr unsigned char kAdjDom = 1;
constexpr unsigned char kAdjMuZero = 2;
struct AdjBuffers {
    void *mu;
    double *self;
    unsigned char *flags;
    unsigned char *status;
};
template <typename Real>
cudaError_t launch_adjoint_fused(const PoolView<Real> &v, const Real *H, const unsigned short *meta,
                                 const double *ih2, const Real *phi, Real *lam, const AdjBuffers &prev,
                                 const AdjBuffers &out, int mode, bool abs_terms, const int *blocks, int nlaunch,
                                 Real rho, double dt, double Dw, double *grad_acc, cudaStream_t s);
// out[b] = 1 when a cell of block b (identity slots) is > 0
template <typename Real>
cudaError_t launch_block_any_positive(const Real *phi, int nblocks, unsigned char *out, cudaStream_t s);
// dL/dphi of loss = -(L_T1c + L_FLAIR) in pool order; roi_count: NULL (every
// voxel once) or how often the ROI lists each voxel of the dense grid
template <typename Real>
cudaError_t launch_loss_grad(int bpd, const Real *phi, const unsigned char *t1c, const unsigned char *flair,
                             const int *roi_count, double t1uc, double t2uc, double slope, Real *lam, cudaStream_t s);
cudaError_t launch_roi_count(int n, const int *roi, int nroi, int *count, cudaStream_t s);
template <typename Real>
cudaError_t launch_gaussian_ic(int bpd, const Real *pw, const Real *pg, const double x0[3], double sigma, Real *out,
                               cudaStream_t s);
template <typename Real>
cudaError_t launch_x0_grad(int bpd, const Real *c0, const Real *lam0, const double x0[3], double sigma,
                           double *partial, int nparts, cudaStream_t s);

template <typename Real>
cudaError_t launch_dense_scatter(const Real *dense, Real *pool, int n, bool to_pool, cudaStream_t s);
// per-CTA partials of the largest p_w * Dw + p_g * Dg and the smallest block
// spacing (partial: 2 * nparts doubles)
template <typename Real>
cudaError_t launch_cfl(const PoolView<Real> &v, Real Dw, Real Dg, double *partial, int nparts, cudaStream_t s);

}  // namespace gbfk
