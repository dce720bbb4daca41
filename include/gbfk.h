/*
 * gbfk -- B200-native Fisher-Kolmogorov reaction-diffusion step on MRAG's
 * block grid (GliomaSolver's RD hot path), C ABI.
 *
 * The reference runs the path as two block sweeps issued by
 * Glioma_ReactionDiffusion::_reactionDiffusionStep
 * (Glioma/Glioma_ReactionDiffusion.cpp:176-187):
 *   blockProcessing.pipeline_process(vInfo, collection, boundaryInfo,
 *                                    ReactionDiffusionOperator<3>(Dw, Dg, rho));
 *   BlockProcessing::process(vInfo, collection, UpdateTumor<3>(dt), gran);
 * with ghost cells reconstructed per block by BlockLab::load
 * (MRAG/MRAGcore/MRAGBlockLab.h:154-301) from BoundaryInfoBlock instruction
 * lists (MRAG/MRAGcore/MRAGBoundaryBlockInfo.h:69-176).  This library keeps
 * the block data resident in GPU memory and replaces those sweeps, the ghost
 * reconstruction, the wavelet detail sweep that drives refinement
 * (MRAG/MRAGcore/MRAGBlockFWT.h:447-478) and the split/collapse data movement
 * (MRAG/MRAGcore/MRAGBlockSplitter.h:24-99, MRAGBlockCollapser.h:22-84).
 * The block tree and the refine/compress planning stay with the caller.
 *
 * Conventions
 *  - Every function returns GBFK_OK (0) or a GBFK_E_* code; the message of
 *    the last failure is gbfk_last_error(ctx).  Nothing aborts.
 *  - A context owns one CUDA stream; calls on one context are serialised by
 *    the caller; different contexts may be used from different threads.
 *  - Work is asynchronous on the context's stream; gbfk_sync waits.
 *  - "Real" is the precision the context was created with: double
 *    (GBFK_F64, the reference built with -D_MRAG_REAL_=double) or float
 *    (GBFK_F32, the reference's default Real, MRAG/MRAGcore/MRAGCommon.h:43-47).
 *    Host buffers passed to upload/download functions hold Real values.
 *  - Block data: 8x8x8 cells per block, x fastest (MRAG/MRAGcore/MRAGBlock.h:40).
 *    A pool "slot" holds one block; cell c of slot s is element s*512 + c.
 */
#ifndef GBFK_H
#define GBFK_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GBFK_BLOCK_SIZE 8
#define GBFK_BLOCK_CELLS 512
#define GBFK_LAB_GHOSTS 488 /* (8+2)^3 - 8^3 ghosts of a lab with stencil [-1,2) */

enum gbfk_status {
    GBFK_OK = 0,
    GBFK_E_INVALID = 1, /* bad argument or call order */
    GBFK_E_CUDA = 2,    /* a CUDA runtime call failed */
    GBFK_E_OOM = 3,     /* device allocation failed or pool too small */
    GBFK_E_NAN = 4,     /* a step produced NaN/Inf in phi */
    GBFK_E_TIMEOUT = 5, /* a bounded device wait gave up */
    GBFK_E_STATE = 6,   /* required data (topology, fields) not uploaded */
    GBFK_E_TOO_LARGE = 7, /* grid larger than gbfk_rd_step_static's fixed scratch */
    GBFK_E_IO = 8         /* a file could not be opened, read or written, or is malformed */
};

enum gbfk_precision { GBFK_F64 = 0, GBFK_F32 = 1 };

/* Fields of the reference's Cell (Glioma/Glioma_Types.h:21-59) that the path uses. */
enum gbfk_field { GBFK_PHI = 0, GBFK_PW = 1, GBFK_PG = 2 };

typedef struct gbfk_ctx gbfk_ctx;

typedef struct {
    int precision;  /* enum gbfk_precision */
    int max_blocks; /* pool capacity in blocks (slots) */
    int device;     /* CUDA device ordinal */
    void *stream;   /* cudaStream_t to use, or NULL for a context-owned stream */
} gbfk_config;

/* One leaf block, as MRAG::BlockInfo (MRAG/MRAGcore/MRAGCommon.h:166-260). */
typedef struct {
    int slot;        /* pool slot holding the block's data */
    int level;       /* BlockInfo::level */
    int index[3];    /* BlockInfo::index */
    double h;        /* BlockInfo::h[0]: grid spacing, 2^-level / 8 */
} gbfk_blockinfo;

/* Ghost reconstruction lists of every block, flattened from
 * BoundaryInfoBlock (MRAGBoundaryBlockInfo.h:69-176).  Block i of the
 * topology owns rows [i*488, (i+1)*488), in the order BlockLab::load visits
 * its ghosts (MRAGBlockLab.h:256-279: codes 0..26 without 13, then z, y, x of
 * the code's region) for the lab range [-1, 9)^3.  Row r's value is
 *   ghost = 0; for k in [row_ptr[r], row_ptr[r+1]): ghost += field[src[k]] * w(k)
 * with w(k) = (Real(w0[k]) * Real(w1[k])) * Real(w2[k]) in Real, exactly as
 * BlockLab::load (MRAGBlockLab.h:286-291).  src[k] = slot * 512 + cell. */
typedef struct {
    int64_t nrows;          /* = nblocks * 488 */
    const int64_t *row_ptr; /* nrows + 1 */
    const int64_t *src;
    const double *w0, *w1, *w2;
} gbfk_ghost_csr;

/* --- context ---------------------------------------------------------- */
/* Replaces the BlockCollection + BlockProcessing objects of the driver
 * (Glioma/Glioma_ReactionDiffusion.h:18-19). */
int gbfk_create(const gbfk_config *cfg, gbfk_ctx **out);
int gbfk_destroy(gbfk_ctx *ctx);
const char *gbfk_last_error(const gbfk_ctx *ctx);
int gbfk_sync(gbfk_ctx *ctx);
/* Kernels this context launched since it was created (a launch counter). */
int64_t gbfk_launch_count(const gbfk_ctx *ctx);

/* --- topology --------------------------------------------------------- */
/* A uniform, periodic bpd^3 grid of one level (MRAG::Grid(bpd,bpd,bpd),
 * MRAG/MRAGcore/MRAGrid.inl:57-111 with periodic ghosts :930-1076); block
 * (bx,by,bz) lives in slot bx + bpd*(by + bpd*bz); h = 1/(8*bpd). */
int gbfk_set_uniform(gbfk_ctx *ctx, int bpd);
/* Any leaf set with its ghost lists (Grid::getBlocksInfo +
 * Grid::getBoundaryInfo, MRAGrid.inl:190-219,514-560). */
int gbfk_set_topology(gbfk_ctx *ctx, const gbfk_blockinfo *blocks, int nblocks,
                      const gbfk_ghost_csr *ghosts);
int gbfk_num_blocks(const gbfk_ctx *ctx);

/* --- data ------------------------------------------------------------- */
/* Copy ncells Real values between host memory and the pool, starting at
 * pool element first_cell (= slot * 512 + cell). */
int gbfk_upload_field(gbfk_ctx *ctx, int field, const void *host, int64_t first_cell,
                      int64_t ncells);
int gbfk_download_field(gbfk_ctx *ctx, int field, void *host, int64_t first_cell,
                        int64_t ncells);
/* Uniform grids only: a dense n^3 volume (x fastest, n = 8*bpd) of Real,
 * scattered into / gathered from the blocks on the device. */
int gbfk_upload_dense(gbfk_ctx *ctx, int field, const void *host, int n);
int gbfk_download_dense(gbfk_ctx *ctx, int field, void *host, int n);

/* --- the hot path ----------------------------------------------------- */
/* nsteps explicit Euler steps: each is ReactionDiffusionOperator<3>(Dw,Dg,rho)
 * over all blocks (Glioma/Operators/ReactionDiffusionOperator.h:47-138)
 * followed by UpdateTumor<3>(dt) (:189-226), fused into one kernel per step
 * (plus a ghost fill of phi where the grid has coarse-fine faces).  Dw, Dg,
 * rho are the rescaled Real values of Glioma_ReactionDiffusion::run
 * (Glioma_ReactionDiffusion.cpp:302-307).  If check_nan is non-zero the call
 * synchronises and returns GBFK_E_NAN when phi became NaN/Inf. */
int gbfk_rd_step(gbfk_ctx *ctx, double Dw, double Dg, double rho, double dt, int nsteps,
                 int check_nan);
/* Which kernel runs the step (no counterpart in the reference: the
 * reference has one CPU operator).  GBFK_STEP_AUTO (the default) runs the
 * persistent TMA-fed pipeline where it applies -- a uniform periodic
 * power-of-two grid from gbfk_set_uniform -- and the one-CTA-per-block kernel
 * elsewhere; all give bit-identical results.  GBFK_STEP_RUN runs the
 * pipeline over all steps of a gbfk_rd_step call in one cooperative launch
 * (the first step alone when phi was uploaded since the last step): each
 * CTA keeps its blocks and, between steps, waits only for the CTAs that
 * own their face neighbours.  On a B200 it is within a few percent of one
 * launch per step (3% faster at 128^3 in FP32, up to 5% slower in FP64),
 * so AUTO does not pick it.  GBFK_STEP_PIPELINED or GBFK_STEP_RUN on a
 * grid they do not apply to make gbfk_rd_step return GBFK_E_STATE.
 * gbfk_step_kernel reports the kernel of the last gbfk_rd_step (0 before
 * any).  A pipeline stage whose copies never complete, or a neighbour that
 * never reports a step, ends its wait after about a second; gbfk_rd_step
 * with check_nan, or gbfk_sync, then returns GBFK_E_TIMEOUT. */
#define GBFK_STEP_AUTO 0
#define GBFK_STEP_BLOCK 1
#define GBFK_STEP_PIPELINED 2
#define GBFK_STEP_RUN 3
int gbfk_set_step_kernel(gbfk_ctx *ctx, int kind);
int gbfk_step_kernel(const gbfk_ctx *ctx);
/* The operator alone: writes dphidt (Real, pool order, nblocks*512 cells) to
 * host memory; phi is unchanged.  (ReactionDiffusionOperator.h:47-138.) */
int gbfk_rd_rhs(gbfk_ctx *ctx, double Dw, double Dg, double rho, void *host_dphidt);
/* CFL time step of the current leaves: the reference's
 *   dt = 0.99 * h*h / (2 * 3 * max(Dw, Dg))   (Glioma_ReactionDiffusion.cpp:306-307)
 * in Real, with h the smallest block spacing of the leaves (the reference's
 * driver takes h of the initial grid, which exceeds the stable step once
 * blocks are refined).  A device reduction (warp shuffles, then per CTA)
 * also finds the largest local coefficient p_w * Dw + p_g * Dg of any cell.
 * out[0] = dt, out[1] = the smallest h, out[2] = the largest coefficient.
 * Dw, Dg: the rescaled coefficients, as for gbfk_rd_step.  Synchronises. */
int gbfk_cfl(gbfk_ctx *ctx, double Dw, double Dg, double out[3]);
/* Host-to-host stepping for solves whose state lives in host memory between
 * calls (one sample after the other, each from its own initial state): phi
 * is copied in from host_in (dense n^3 Real, x fastest, n = 8*bpd, uniform
 * grids only), advanced nsteps steps as by gbfk_rd_step, and copied out to
 * host_out.  Asynchronous: the copies run on two internal streams with two
 * sets of staging buffers, so that the output copy of one call overlaps the
 * input copy of the next (PCIe carries both directions at once).  host_in
 * and host_out must stay untouched until gbfk_sync (pinned buffers give the
 * overlap; pageable ones are copied synchronously).  gbfk_join_copies makes
 * the context's stream wait for every copy issued so far, so that work or
 * events recorded on it afterwards follow them; gbfk_sync joins and waits.
 * NaN is not checked here (use gbfk_rd_step with check_nan). */
int gbfk_rd_step_host(gbfk_ctx *ctx, const void *host_in, void *host_out, double Dw, double Dg, double rho,
                      double dt, int nsteps);
int gbfk_join_copies(gbfk_ctx *ctx);

/* --- adaptivity ------------------------------------------------------- */
/* Per block of the topology (in upload order) the max |detail| of the
 * one-level interpolating-wavelet transform of phi, as
 * FWTReport::getOverAll_DetailMaxMag after BlockFWT::multichannel_fwt<0,0>
 * (MRAG/MRAGcore/MRAGBlockFWT.h:109-120,219-298,447-478).  out: nblocks doubles. */
int gbfk_fwt_details(gbfk_ctx *ctx, double *out);
/* Split nsplit parents into 8 children each by Hs synthesis
 * (BlockSplitter::_splitBlocks, MRAGBlockSplitter.h:24-99), all three fields.
 * parents[i] is a block index of the current topology (its lab ghosts are
 * used); children[8*i + c] is the destination slot of child
 * c = cx + 2*(cy + 2*cz).  Destination slots must not hold current blocks. */
int gbfk_split(gbfk_ctx *ctx, int nsplit, const int *parents, const int *children);
/* Collapse ncollapse groups of 8 sibling slots into one parent slot by Ha
 * analysis (injection; BlockCollapser::_collapseBlocks, MRAGBlockCollapser.h:
 * 22-84).  children[8*i + c] as for gbfk_split; parents[i] is a slot. */
int gbfk_collapse(gbfk_ctx *ctx, int ncollapse, const int *children, const int *parents);

/* --- batched TMCMC-stage forward solves --------------------------------- */
/* The reference evaluates the samples of a TMCMC stage as independent tasks
 * (tools/pi4u_lite/Inference/engine_tmcmc.c:597-624), each a separate solver
 * process (tools/pi4u_lite/Inference/fitfun_glioma.c:46-245).  A batch keeps
 * every sample of a stage in GPU memory and advances all samples that have
 * not reached their own horizon with one launch per time step. */
typedef struct gbfk_batch gbfk_batch;
/* Initial conditions of a batch sample.  GBFK_IC_BALL is the reference's
 * tumour of Glioma_ReactionDiffusion::_ic (Glioma_ReactionDiffusion.cpp:
 * 155-164), the ball of radius 0.005 smoothed over a width of 1/64 around x0
 * (x0 rounded to Real), where the cell has tissue; its values are computed
 * on the host in the reference's arithmetic (only the cells near x0) and
 * scattered into the zeroed state on the device, so they equal
 * gbfk_map_anatomy's phi bit for bit.  The reference's inner core
 * (psi < -1) is empty for that radius and width, and its band test
 * pGM + pWM > 0 is p_w + p_g > 0 for non-negative fractions. */
enum gbfk_ic { GBFK_IC_GAUSSIAN = 0, GBFK_IC_BALL = 1 };
typedef struct {
    double Dw, Dg, rho; /* rescaled Real coefficients, as for gbfk_rd_step */
    double dt;          /* time step */
    int nsteps;         /* steps to this sample's horizon */
    int anatomy;        /* which anatomy (gbfk_batch_set_anatomy) */
    double x0[3];       /* tumour origin in the unit cube */
    double sigma;       /* GBFK_IC_GAUSSIAN: c0 = exp(-|x-x0|^2/(2 sigma^2)) where p_w+p_g > 0 */
    int ic;             /* enum gbfk_ic: the initial condition around x0 */
} gbfk_sample;
/* A batch on a uniform periodic bpd^3 grid with room for max_samples samples
 * and max_anatomies anatomies (2 phi buffers + face coefficients per sample). */
int gbfk_batch_create(const gbfk_config *cfg, int bpd, int max_samples, int max_anatomies, gbfk_batch **out);
int gbfk_batch_destroy(gbfk_batch *b);
const char *gbfk_batch_last_error(const gbfk_batch *b);
int64_t gbfk_batch_launch_count(const gbfk_batch *b);
/* p_w, p_g of one anatomy: dense n^3 Real volumes (x fastest, n = 8*bpd). */
int gbfk_batch_set_anatomy(gbfk_batch *b, int anatomy, const void *pw_dense, const void *pg_dense);
int gbfk_batch_set_samples(gbfk_batch *b, int nsamples, const gbfk_sample *samples);
/* Build every sample's initial condition and face coefficients, then run all
 * samples to their horizons.  samples_per_cta: -1 for the persistent
 * pipelined step over all active samples (a power-of-two bpd only), 1, 2 or
 * 4 for the one-CTA-per-block kernel with that many samples per CTA, or 0 to
 * let the autotuner time the candidates on the first steps and keep the
 * fastest (the results do not depend on it).  GBFK_E_NAN if a sample became
 * NaN; GBFK_E_STATE for -1 on a grid it does not apply to. */
int gbfk_batch_run(gbfk_batch *b, int samples_per_cta);
/* The samples_per_cta choice the last run used (-1: the pipelined step). */
int gbfk_batch_samples_per_cta(const gbfk_batch *b);
/* The launch shape of the pipelined step the last run used: consumer warps
 * per CTA, heavy-block ring slots, empty-block ring slots (all 0 when it
 * used the per-block kernel).  With samples_per_cta 0 the autotuner times
 * every compiled shape; otherwise the shape is the default (or the
 * GBFK_TMA_SHAPE="warps,heavy,empty" environment variable). */
int gbfk_batch_tile_shape(const gbfk_batch *b, int shape[3]);
/* gbfk_batch_run replays its steps after the autotuner and the first step as
 * CUDA graphs of up to 512 launches captured on the batch's stream; this is
 * how many the last run replayed (0 when the stream could not be captured,
 * e.g. the legacy default stream). */
int gbfk_batch_graph_count(const gbfk_batch *b);
/* phi of one sample after the run, dense n^3 Real. */
int gbfk_batch_download(gbfk_batch *b, int sample, void *dense_out);

/* --- UQ: finest-uniform dump and likelihood ---------------------------- */
/* Parameters of the likelihood (LikelihoodInput.txt and the -stepPET /
 * -stepMRI flags of tools/pi4u_lite/Inference/Likelihood/source/HGG_Likelihood.cpp:11-36). */
typedef struct {
    double pet_sigma2, pet_scale; /* PET Gaussian: variance, signal scale */
    double t1_uc, t2_uc, slope;   /* T1c / FLAIR thresholds, sigmoid slope */
    int step_pet, step_mri;       /* sub-sampling steps */
} gbfk_likelihood_params;
/* Observations on the n^3 dump grid (x fastest): T1c and FLAIR masks (a voxel
 * counts as 1 where the value equals 1), the PET signal (NULL: no PET term),
 * and the ROI voxel list of -bROI 1 (nroi (x,y,z) triples; NULL: every voxel;
 * HGG_Likelihood.cpp:97-124). */
int gbfk_set_observations(gbfk_ctx *ctx, int n, const double *t1c, const double *flair, const double *pet,
                          const int *roi, int nroi);
/* Glioma_ReactionDiffusion::_dumpUQoutput (Glioma_ReactionDiffusion.cpp:208-262):
 * phi written onto the n^3 grid of the initial resolution (n = 8 * initial
 * blocks per direction), as doubles, x fastest, to host memory. */
int gbfk_uq_dump(gbfk_ctx *ctx, int n, double *host_out);
/* The log-likelihood of the current phi against the observations
 * (HGG_Likelihood::run, HGG_Likelihood.cpp:176-192): out[0] = PET,
 * out[1] = T1c, out[2] = FLAIR, out[3] = their sum (the reference writes
 * -out[3] to Likelihood.txt).  Sums are FP64 with compensation. */
int gbfk_log_likelihood(gbfk_ctx *ctx, const gbfk_likelihood_params *params, double out[4]);
/* The likelihood step of every sample after the run, on the device: in the
 * reference each TMCMC sample dumps its state to a file
 * (Glioma_ReactionDiffusion.cpp:208-262) and a separate likelihood process
 * reads it (HGG_Likelihood::run, HGG_Likelihood.cpp:176-192).  Observations
 * as for gbfk_set_observations, on the batch's n^3 grid, shared by all
 * samples; gbfk_batch_log_likelihood writes out[4 * s .. 4 * s + 3] =
 * PET, T1c, FLAIR and their sum for sample s (the caller's order), with
 * params[0] for every sample or, if per_sample, params[s] (a TMCMC sample
 * carries its own PET and threshold parameters, fitfun_glioma.c:128-151).
 * The grid is uniform, so the dump is the samples' own cells.  After a run
 * that reported GBFK_E_NAN the values of the NaN samples are NaN. */
int gbfk_batch_set_observations(gbfk_batch *b, const double *t1c, const double *flair, const double *pet,
                                const int *roi, int nroi);
int gbfk_batch_log_likelihood(gbfk_batch *b, const gbfk_likelihood_params *params, int per_sample, double *out);

/* --- discrete adjoint ------------------------------------------------- */
/* No counterpart in the reference (which samples with TMCMC and never
 * differentiates).  Forward solve plus the hand-written discrete adjoint of
 * the fused step on the context's uniform grid, for the loss
 *   loss = -(L_T1c + L_FLAIR)        (HGG_Likelihood.cpp:77-156)
 * of the state at the horizon against the observations (gbfk_set_observations;
 * with a ROI the sums run over its points, each as often as it is listed,
 * as the likelihood's -bROI does, HGG_Likelihood.cpp:97-124).  dt and the step count are held fixed; the piecewise-constant
 * switches of the step (domain test, no-flux doubling, clamp) are held fixed.
 * States are kept with binomial checkpointing in nsnapshots device buffers;
 * these and seven work fields stay allocated in the context until
 * gbfk_destroy, so that later calls on the same grid with at most as many
 * checkpoints allocate nothing.  The forward steps of the reverse sweep run
 * on a second stream of the context (created at the first call, ordered
 * after the work already on the context's stream) next to the adjoint steps;
 * the call returns when both are done.  GBFK_ADJ_STREAMS=1 keeps everything
 * on the context's stream (the same results). */
typedef struct {
    double Dw, Dg, rho, dt; /* rescaled Real coefficients and the time step */
    int nsteps;             /* steps to the horizon */
    int nsnapshots;         /* checkpoint buffers (>= 1) */
    double x0[3];           /* tumour origin, used when sigma > 0 */
    double sigma;           /* > 0: c0 = exp(-|x-x0|^2/(2 sigma^2)) where p_w+p_g > 0;
                               <= 0: c0 = the context's current phi */
    double t1_uc, t2_uc, slope; /* Bernoulli loss parameters */
    int flags;              /* 0, or GBFK_ADJ_TERM_MAGNITUDES */
} gbfk_adjoint_params;
/* Also sum the magnitudes of the terms of dDw and drho (one per domain cell
 * and step): |dDw| / dDw_abs near 0 means the terms cancel, and a relative
 * change e of the terms (the rounding of FP32 states) can move dDw by up to
 * e * dDw_abs. */
#define GBFK_ADJ_TERM_MAGNITUDES 1
typedef struct {
    double loss;            /* -(L_T1c + L_FLAIR) at the horizon */
    double dDw, drho;       /* d loss / d Dw (with Dg = 0.1 Dw), d loss / d rho */
    double dx0[3];          /* d loss / d x0 (0 when sigma <= 0) */
    int64_t forward_steps;  /* forward steps run, recomputation included */
    int64_t adjoint_steps;
    double dDw_abs, drho_abs; /* with GBFK_ADJ_TERM_MAGNITUDES: the sums of the terms' magnitudes; else 0 */
} gbfk_adjoint_result;
/* grad_c0_dense: NULL, or n^3 Real (x fastest) receiving d loss / d c0. */
int gbfk_forward_adjoint(gbfk_ctx *ctx, const gbfk_adjoint_params *params, gbfk_adjoint_result *out,
                         void *grad_c0_dense);

/* --- patient data: Matrix files and the anatomy mapping ---------------- */
/* Host-only functions (no GPU, no context).  Their failure message is
 * gbfk_host_last_error(), kept per calling thread. */
const char *gbfk_host_last_error(void);
/* The reference's Matrix file (Glioma/Matrix.h:20-34,71-88,141-240 and the
 * D2D/D3D dump/load at :390-445,609-665; the likelihood program reads the
 * same layout through its own copy of Matrix.h): int32 1234 (the magic
 * number; a byte-swapped file fails it), int32 dim (2 or 3), dim int32
 * sizes (x first), int32 type id (0 double, 1 float, 2 int32), then the
 * values, x fastest.  gbfk_matrix_info reads the header; sizes[d] = 1 for
 * d >= dim.  GBFK_E_IO for a missing file, a short read, a wrong magic
 * number, a dim other than 2 or 3, a negative size or an unknown type id
 * (the reference prints a message and keeps an unusable matrix). */
int gbfk_matrix_info(const char *path, int *dim, int sizes[3], int *type_id);
/* All values converted to double, as MatrixD2D/MatrixD3D<double> load them
 * (Matrix.h:116-169): capacity must hold sizes[0]*sizes[1]*sizes[2] values. */
int gbfk_matrix_read(const char *path, double *out, int64_t capacity);
/* Writes data (sizes[0]*...*sizes[dim-1] doubles, x fastest) with the given
 * type id (Matrix.h:184-240): float rounds to nearest, int32 truncates
 * towards zero and rejects values outside int32 (GBFK_E_INVALID). */
int gbfk_matrix_write(const char *path, int dim, const int *sizes, int type_id, const double *data);
/* Glioma_ReactionDiffusion::_ic (Glioma/Glioma_ReactionDiffusion.cpp:79-172)
 * on the uniform bpd^3-block grid the reference constructs before its first
 * refinement: for each cell at vertex position x (BlockInfo::pos,
 * MRAG/MRAGcore/MRAGCommon.h:199-205) the anatomy voxel floor(x / (1/M)),
 * M = max(msize), is mapped when it lies inside the volumes (all fields stay
 * 0 elsewhere, the Cell defaults of Glioma/Glioma_Types.h:54-77); CSF wins
 * the majority vote against p_w + p_g (:144-147), p_w and p_g are then
 * normalised by the remaining tissue (:149-151), and the tumour is the
 * smoothed ball of radius 0.005 and width 1/64 around tumor_ic (:157-164).
 *   gm, wm, csf : msize[0] x msize[1] x msize[2] doubles, x fastest (the
 *                 MatrixD3D files {prefix}GM.dat, WM.dat, CSF.dat);
 *   tumor_ic    : tumour centre in the unit cube, rounded to Real;
 *   pw, pg, pcsf, phi : NULL or dense (8*bpd)^3 Real outputs, x fastest;
 *   tissue      : NULL or dense (8*bpd)^3 Real: p_w + p_g after the vote and
 *                 before the normalisation (the tumour's tissue test);
 *   L           : NULL or the characteristic length M * 0.1 (cm) in Real.
 * Arithmetic follows the reference in its Real (GBFK_F64: double; GBFK_F32:
 * float, with the mixed float/double expressions of the reference's default
 * build), so the outputs are bit-identical to the reference's cells.  Runs
 * on host threads over z-planes. */
int gbfk_map_anatomy(int precision, int bpd, const int msize[3], const double *gm, const double *wm,
                     const double *csf, const double tumor_ic[3], void *pw, void *pg, void *pcsf, void *phi,
                     void *tissue, double *L);

/* --- failure detection ------------------------------------------------ */
/* No counterpart in the reference.  Checks on `device` that the bounded wait
 * of the pipelined step gives up instead of hanging: a one-thread kernel
 * waits for an mbarrier phase that nothing completes, the wait ends after its
 * limit (1 s of device time) and the kernel records it, as a step records a
 * copy that never landed.  Returns GBFK_E_TIMEOUT (what gbfk_rd_step reports
 * for such a step) with the seconds the kernel took; GBFK_OK would mean the
 * phase completed, GBFK_E_CUDA a failed CUDA call.  The device stays usable. */
int gbfk_probe_bounded_wait(int device, double *seconds);

/* --- allocation-free step -------------------------------------------- */
/* No counterpart in the reference.  One fused RD step (the operator and the
 * update of gbfk_rd_step) on a uniform periodic bpd^3 grid, for callers that
 * cannot let the library call cudaMalloc: code whose device memory belongs to
 * another allocator that reserved it up front, or a time loop that must not
 * pay cudaMalloc's device-wide synchronisation.  It allocates nothing and
 * frees nothing: its scratch (face coefficients, meta words, block types,
 * neighbour table) is one fixed device array of about 7.3 MiB that every GPU
 * loading the library holds until the process exits.
 *   pw, pg, phi_in : device arrays of bpd^3 * 512 Real in block-pool order
 *                    (block (bx,by,bz) at slot bx + bpd*(by + bpd*bz));
 *   phi_out        : device array of the same size that overlaps phi_in
 *                    nowhere (GBFK_E_INVALID otherwise);
 *   Dw, Dg, rho, dt: as for gbfk_rd_step; stream: a cudaStream_t of `device`
 *                    (GBFK_E_INVALID for another device's stream) or NULL for
 *                    the legacy default stream; device: CUDA ordinal.
 * Returns GBFK_E_TOO_LARGE when bpd^3 > GBFK_STATIC_MAX_BLOCKS.  Every call
 * on a device shares the scratch array (it keeps the last call's contents and
 * is fully rewritten by each call), so calls that overlap on the GPU race:
 * serialise them.  The first call on a device (and the first after its
 * context was reset) looks up the array's address with that device current;
 * make it before any stream capture.  The work is asynchronous on the stream.
 * No NaN check: a step that produces NaN or Inf still returns GBFK_OK (check
 * the output where that matters).  The caller's current device is restored;
 * an error the caller's earlier work left pending is returned as GBFK_E_CUDA
 * and left in place. */
#define GBFK_STATIC_MAX_BLOCKS 512
int gbfk_rd_step_static(int precision, int bpd, const void *pw, const void *pg, const void *phi_in,
                        void *phi_out, double Dw, double Dg, double rho, double dt, void *stream,
                        int device);

#ifdef __cplusplus
}
#endif
#endif /* GBFK_H */
