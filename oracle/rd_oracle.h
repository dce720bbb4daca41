/*
 * CPU restatement of GliomaSolver's Fisher-Kolmogorov path (the oracle).
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may load this library, and only as the checker
 * or the timed CPU baseline.  The product (libgbfk) never calls it.
 *
 * Every function restates the reference's arithmetic operation by operation,
 * in the reference's Real type, so that results can be compared bit for bit:
 *   *_f64  = reference built with -D_MRAG_REAL_=double
 *   *_f32  = reference default build (Real = float, MRAGCommon.h:43-47), in
 *            which the operator still evaluates ih2, the harmonic-mean
 *            quotient, the flux sums and the reaction term in double
 *            (Glioma/Operators/ReactionDiffusionOperator.h:49-52,124-135).
 * The restatement is pinned against the reference itself: oracle/_ref is the
 * reference's own operator code (oracle/ref_harness.cpp), and the golden
 * fixtures under tests/golden/ were produced by it.
 *
 * Layouts
 *   dense  : n^3 cells, x fastest, periodic wrap (the uniform MRAG grid with
 *            periodic ghosts, MRAG/MRAGcore/MRAGrid.inl:37-39,930-1076).
 *   pool   : nblocks x 512 cells (8^3 block, x fastest, MRAGBlock.h:40) plus a
 *            per-block lab halo of 488 ghost cells filled from a ghost CSR
 *            (the instruction lists of MRAGBoundaryBlockInfo.h:69-176, as
 *            executed by BlockLab::load, MRAGBlockLab.h:254-295).
 */
#ifndef GBFK_RD_ORACLE_H
#define GBFK_RD_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* dphidt of one ReactionDiffusionOperator<3> sweep on a dense periodic grid
 * (ReactionDiffusionOperator.h:97-138). */
void orc_rd_rhs_dense_f64(int n, const double *pw, const double *pg, const double *phi,
                          double Dw, double Dg, double rho, double h, double *dphidt);
void orc_rd_rhs_dense_f32(int n, const float *pw, const float *pg, const float *phi,
                          float Dw, float Dg, float rho, float h, float *dphidt);

/* nsteps explicit Euler steps (operator + UpdateTumor, ReactionDiffusionOperator.h:
 * 189-226) on a dense periodic grid, in place on phi; scratch holds n^3 Reals. */
void orc_rd_steps_dense_f64(int n, const double *pw, const double *pg, double *phi,
                            double Dw, double Dg, double rho, double h, double dt, int nsteps,
                            double *scratch);
void orc_rd_steps_dense_f32(int n, const float *pw, const float *pg, float *phi,
                            float Dw, float Dg, float rho, float h, double dt, int nsteps,
                            float *scratch);

/* Ghost CSR: one row per lab ghost cell of each block, rows ordered block by
 * block, and inside a block by BlockLab::load's loop order (codes 0..26 without
 * 13, then z, y, x of the code's region, MRAGBlockLab.h:256-279) for the lab
 * range [-1, 9) in every direction (the grid's max stencil [-1, 2),
 * MRAG/MRAGcore/MRAGrid.inl:761-789), i.e. 488 rows per block.  Entry k of a
 * row reads cell src[k] (= source block slot * 512 + cell index) with the
 * three weights w0[k], w1[k], w2[k] (doubles of BoundaryInfoBlock::weightsPool). */
typedef struct {
    int64_t nrows;
    const int64_t *row_ptr;   /* nrows + 1 */
    const int64_t *src;
    const double *w0, *w1, *w2;
} orc_ghost_csr;

#define ORC_LAB_GHOSTS 488

/* Fill the lab ghosts of every block for one field (BlockLab::load step 3:
 * ghost = 0; ghost += v * ((w0*w1)*w2), in Real). out: nblocks * 488. */
void orc_fill_ghosts_f64(const orc_ghost_csr *g, const double *field, double *out);
void orc_fill_ghosts_f32(const orc_ghost_csr *g, const float *field, float *out);

/* One operator sweep (+ optional update) over a block pool with lab ghosts.
 * h[b] is BlockInfo::h[0] of block b (in Real). */
void orc_rd_rhs_pool_f64(int nblocks, const double *h, const double *pw, const double *pg,
                         const double *phi, const double *gpw, const double *gpg,
                         const double *gphi, double Dw, double Dg, double rho, double *dphidt);
void orc_rd_rhs_pool_f32(int nblocks, const float *h, const float *pw, const float *pg,
                         const float *phi, const float *gpw, const float *gpg,
                         const float *gphi, float Dw, float Dg, float rho, float *dphidt);
void orc_update_f64(int64_t ncells, double *phi, const double *dphidt, double dt);
void orc_update_f32(int64_t ncells, float *phi, const float *dphidt, double dt);

/* Max |detail| of the one-level interpolating-wavelet transform of phi per
 * block (BlockFWT::_fwt/_filter + FWTReport::getOverAll_DetailMaxMag,
 * MRAG/MRAGcore/MRAGBlockFWT.h:109-120,219-298). out: nblocks doubles. */
void orc_fwt_detail_pool_f64(int nblocks, const double *phi, const double *gphi, double *out);
void orc_fwt_detail_pool_f32(int nblocks, const float *phi, const float *gphi, double *out);

/* Children of a block by Hs synthesis (BlockSplitter::_splitBlocks,
 * MRAG/MRAGcore/MRAGBlockSplitter.h:24-99): child[c] for c = cx + 2*(cy + 2*cz)
 * gets 512 cells; reads the parent's lab (interior + ghosts). */
void orc_split_block_f64(const double *parent, const double *gparent, double *children);
void orc_split_block_f32(const float *parent, const float *gparent, float *children);

/* Parent of eight siblings by Ha analysis (injection; BlockCollapser::
 * _collapseBlocks, MRAG/MRAGcore/MRAGBlockCollapser.h:22-84). */
void orc_collapse_blocks_f64(const double *children, double *parent);
void orc_collapse_blocks_f32(const float *children, float *parent);

/* _dumpUQoutput (Glioma/Glioma_ReactionDiffusion.cpp:208-262): phi of every
 * block written onto the gpd^3 grid of the initial resolution, x fastest.
 * Block b has level[b], index[3*b..], spacing h[b] (Real); cells at
 * x = origin + h*i with origin = index * 2^-level.  Cells of blocks as fine
 * as the dump grid or finer write their voxel (the last cell in loop order
 * wins); coarser blocks write c^3 copies, c = 2, 3 or 4 by h (as the
 * reference).  out must hold gpd^3 doubles and is zeroed first. */
void orc_uq_dump_f64(int nblocks, const int *level, const int *index, const double *h, const double *phi,
                     int gpd, double *out);
void orc_uq_dump_f32(int nblocks, const int *level, const int *index, const float *h, const float *phi,
                     int gpd, double *out);

/* HGG_Likelihood (tools/pi4u_lite/Inference/Likelihood/source/HGG_Likelihood.cpp:
 * 40-156) in long double: out[0] = PET log-likelihood (or 0 if pet is NULL),
 * out[1] = T1c, out[2] = FLAIR; roi (npoints triples) selects voxels for the
 * MRI terms (-bROI 1), NULL = every voxel. */
void orc_log_likelihood(int n, const double *model, const double *t1c, const double *flair, const double *pet,
                        const int *roi, int nroi, double pet_sigma2, double pet_scale, double t1uc,
                        double t2uc, double slope, int step_pet, int step_mri, long double out[3]);

/* Glioma_ReactionDiffusion::_ic (Glioma/Glioma_ReactionDiffusion.cpp:79-172)
 * on the uniform grid of bpd blocks per direction (level ceil(log2 bpd),
 * MRAG/MRAGcore/MRAGridHelpers.h:9-17), n = 8*bpd cells per direction, cell
 * positions x = i * 2^-level / 8.  gm, wm, csf: sx*sy*sz doubles, x fastest
 * (MatrixD3D).  Outputs (n^3 Real each, x fastest, any may be NULL): p_w,
 * p_g, p_csf, phi and the tissue sum p_g + p_w after the vote that the
 * tumour test uses.  Cells whose voxel lies outside the volumes stay 0. */
void orc_map_anatomy_f64(int bpd, int sx, int sy, int sz, const double *gm, const double *wm, const double *csf,
                         const double tumor_ic[3], double *pw, double *pg, double *pcsf, double *phi,
                         double *tissue);
void orc_map_anatomy_f32(int bpd, int sx, int sy, int sz, const double *gm, const double *wm, const double *csf,
                         const double tumor_ic[3], float *pw, float *pg, float *pcsf, float *phi, float *tissue);

/* One step of the discrete adjoint of the fused step, FP64, dense periodic
 * grid (switches held fixed; see rd_oracle.c): lam holds dL/dphi' on entry,
 * dL/dphi on exit; grad[0] += dL/drho, grad[1] += dL/dDw (Dg = 0.1 Dw),
 * grad[2], grad[3] += the magnitudes of those terms; scratch: 8 n^3 doubles. */
void orc_adjoint_step_dense_f64(int n, const double *pw, const double *pg, const double *phi, double Dw,
                                double Dg, double rho, double h, double dt, double *lam, double grad[4],
                                double *scratch);
/* dL/du of loss = -(L_T1c + L_FLAIR) (HGG_Likelihood.cpp:136-156). */
void orc_loss_grad_f64(int64_t ncells, const double *u, const double *t1c, const double *flair, double t1uc,
                       double t2uc, double slope, double *lam);

#ifdef __cplusplus
}
#endif
#endif
