"""Host-side mirror of the reference's operator interface over the C ABI.

The reference drives its RD step through MRAG's block-processing contract
(Glioma/Glioma_ReactionDiffusion.cpp:176-187):

    ReactionDiffusionOperator<_DIM> rhs(Dw, Dg, rho);
    UpdateTumor<_DIM>               updateTumor(dt);
    blockProcessing.pipeline_process(vInfo, collection, *boundaryInfo, rhs);
    BlockProcessing::process(vInfo, collection, updateTumor, nParallelGranularity);

This module keeps those names and argument meanings
(``ReactionDiffusionOperator``, ``UpdateTumor``, ``BlockProcessing.
pipeline_process`` / ``process``) on top of a device-resident ``BlockPool``
(the B200 stand-in for ``BlockCollection`` + ``BoundaryInfo``).  The
operator sweep only records its coefficients; the following update launches
one fused kernel that does both, which is equivalent because the reference
computes every ``dphidt`` before it updates any ``phi``.

Errors: the reference asserts/aborts; here every failure raises
``GbfkError`` with the library's status code and message.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import GbfkError
from .schedule import BLOCK_SIZE

BLOCK_CELLS = BLOCK_SIZE ** 3
LAB_GHOSTS = 488
FIELDS = {"phi": _lib.GBFK_PHI, "p_w": _lib.GBFK_PW, "p_g": _lib.GBFK_PG}


def _ptr(a: np.ndarray):
    if not a.flags.c_contiguous:
        raise ValueError("arrays passed to the C ABI must be C-contiguous")
    return a.ctypes.data_as(ctypes.c_void_p)


class BlockPool:
    """A gbfk context: the device block pool of one solve.

    ``precision`` is the reference build's Real: ``"f64"`` (``-D_MRAG_REAL_=
    double``) or ``"f32"`` (the default float build).
    """

    def __init__(self, max_blocks: int, precision: str = "f64", device: int = 0, stream=None):
        self.lib = _lib.load()
        self.precision = precision
        self.dtype = np.float64 if precision == "f64" else np.float32
        self._io_keep = []  # host buffers of rd_step_host calls not yet synced
        cfg = _lib.Config(_lib.GBFK_F64 if precision == "f64" else _lib.GBFK_F32, int(max_blocks),
                          int(device), stream)
        h = ctypes.c_void_p()
        rc = self.lib.gbfk_create(ctypes.byref(cfg), ctypes.byref(h))
        if rc != _lib.GBFK_OK:
            raise GbfkError(rc, "gbfk_create failed")
        self.ctx = h
        self.max_blocks = int(max_blocks)
        self.n = None  # dense extent of a uniform grid

    # -- plumbing ---------------------------------------------------------
    def _check(self, rc: int):
        if rc != _lib.GBFK_OK:
            msg = self.lib.gbfk_last_error(self.ctx)
            raise GbfkError(rc, msg.decode() if msg else "")

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.gbfk_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def launches(self) -> int:
        return int(self.lib.gbfk_launch_count(self.ctx))

    @property
    def num_blocks(self) -> int:
        return int(self.lib.gbfk_num_blocks(self.ctx))

    def sync(self):
        self._check(self.lib.gbfk_sync(self.ctx))
        self._io_keep.clear()

    # -- topology ---------------------------------------------------------
    def set_uniform(self, blocks_per_dim: int):
        self._check(self.lib.gbfk_set_uniform(self.ctx, int(blocks_per_dim)))
        self.n = BLOCK_SIZE * int(blocks_per_dim)

    def set_topology(self, blocks, csr: dict):
        """``blocks``: sequence of ``(slot, level, (ix, iy, iz), h)``;
        ``csr``: ``row_ptr, src`` (int64) and ``w0, w1, w2`` (float64) of the
        lab ghost lists, 488 rows per block in BlockLab::load order."""
        arr = (_lib.BlockInfo * len(blocks))()
        for i, (slot, level, idx, h) in enumerate(blocks):
            arr[i].slot, arr[i].level, arr[i].h = int(slot), int(level), float(h)
            arr[i].index[0], arr[i].index[1], arr[i].index[2] = (int(v) for v in idx)
        keep = [np.ascontiguousarray(csr[k], dtype=dt) for k, dt in
                (("row_ptr", np.int64), ("src", np.int64), ("w0", np.float64), ("w1", np.float64),
                 ("w2", np.float64))]
        g = _lib.GhostCSR(keep[0].size - 1, *(_ptr(a).value for a in keep))
        self._check(self.lib.gbfk_set_topology(self.ctx, arr, len(blocks), ctypes.byref(g)))
        self.n = None

    # -- data -------------------------------------------------------------
    def upload(self, field: str, values: np.ndarray, first_cell: int = 0):
        a = np.ascontiguousarray(values, dtype=self.dtype).ravel()
        self._check(self.lib.gbfk_upload_field(self.ctx, FIELDS[field], _ptr(a), int(first_cell), a.size))
        self.sync()

    def download(self, field: str, ncells: int, first_cell: int = 0) -> np.ndarray:
        out = np.empty(int(ncells), dtype=self.dtype)
        self._check(self.lib.gbfk_download_field(self.ctx, FIELDS[field], _ptr(out), int(first_cell),
                                                 out.size))
        return out

    def upload_dense(self, field: str, volume: np.ndarray):
        a = np.ascontiguousarray(volume, dtype=self.dtype)
        self._check(self.lib.gbfk_upload_dense(self.ctx, FIELDS[field], _ptr(a), a.shape[0]))
        self.sync()

    def download_dense(self, field: str) -> np.ndarray:
        n = self.n
        out = np.empty((n, n, n), dtype=self.dtype)
        self._check(self.lib.gbfk_download_dense(self.ctx, FIELDS[field], _ptr(out), n))
        return out

    # -- hot path ---------------------------------------------------------
    @property
    def step_kernel(self) -> str:
        """Kernel of the last rd_step: "pipelined" (persistent TMA pipeline,
        uniform power-of-two grids, one launch per step), "run" (the same
        pipeline over all steps of the call in one launch), "block" (one CTA
        per block) or "" before any step.  Assign "auto", "block",
        "pipelined" or "run" to choose."""
        k = int(self.lib.gbfk_step_kernel(self.ctx))
        return {v: n for n, v in _lib.STEP_KERNELS.items()}.get(k, "") if k else ""

    @step_kernel.setter
    def step_kernel(self, kind: str):
        self._check(self.lib.gbfk_set_step_kernel(self.ctx, _lib.STEP_KERNELS[kind]))

    def rd_step(self, Dw, Dg, rho, dt, nsteps: int = 1, check_nan: bool = False):
        self._check(self.lib.gbfk_rd_step(self.ctx, float(Dw), float(Dg), float(rho), float(dt),
                                          int(nsteps), int(bool(check_nan))))

    def rd_rhs(self, Dw, Dg, rho) -> np.ndarray:
        out = np.empty(self.num_blocks * BLOCK_CELLS, dtype=self.dtype)
        self._check(self.lib.gbfk_rd_rhs(self.ctx, float(Dw), float(Dg), float(rho), _ptr(out)))
        return out

    def rd_step_host(self, phi_in: np.ndarray, phi_out: np.ndarray, Dw, Dg, rho, dt, nsteps: int = 1):
        """Asynchronous host-to-host steps (gbfk_rd_step_host): phi_in (dense
        n^3) in, nsteps steps, phi out into phi_out.  Both arrays are kept
        alive here and must stay untouched until sync()."""
        for a in (phi_in, phi_out):
            if a.dtype != self.dtype or not a.flags["C_CONTIGUOUS"]:
                raise ValueError("phi_in and phi_out must be C-contiguous arrays of the pool's Real")
        self._io_keep.extend((phi_in, phi_out))
        self._check(self.lib.gbfk_rd_step_host(self.ctx, _ptr(phi_in), _ptr(phi_out), float(Dw), float(Dg),
                                               float(rho), float(dt), int(nsteps)))

    def join_copies(self):
        """Make the pool's stream wait for the copies of rd_step_host."""
        self._check(self.lib.gbfk_join_copies(self.ctx))

    def cfl(self, Dw, Dg) -> dict:
        """The reference's CFL step at the finest leaf spacing, the smallest
        spacing and the largest local coefficient p_w Dw + p_g Dg (gbfk_cfl)."""
        out = np.empty(3, dtype=np.float64)
        self._check(self.lib.gbfk_cfl(self.ctx, float(Dw), float(Dg), _ptr(out)))
        return {"dt": float(out[0]), "h_min": float(out[1]), "max_diffusion": float(out[2])}

    # -- adaptivity -------------------------------------------------------
    def fwt_details(self) -> np.ndarray:
        out = np.empty(self.num_blocks, dtype=np.float64)
        self._check(self.lib.gbfk_fwt_details(self.ctx, _ptr(out)))
        return out

    def split(self, parents, children):
        p = np.ascontiguousarray(parents, dtype=np.int32)
        c = np.ascontiguousarray(children, dtype=np.int32).ravel()
        if c.size != 8 * p.size:
            raise ValueError("split needs 8 child slots per parent")
        self._check(self.lib.gbfk_split(self.ctx, p.size, _ptr(p), _ptr(c)))

    def collapse(self, children, parents):
        p = np.ascontiguousarray(parents, dtype=np.int32)
        c = np.ascontiguousarray(children, dtype=np.int32).ravel()
        if c.size != 8 * p.size:
            raise ValueError("collapse needs 8 child slots per parent")
        self._check(self.lib.gbfk_collapse(self.ctx, p.size, _ptr(c), _ptr(p)))


    # -- UQ -----------------------------------------------------------------
    def uq_dump(self, n: int) -> np.ndarray:
        """phi on the n^3 grid of the initial resolution (_dumpUQoutput)."""
        out = np.empty((n, n, n), dtype=np.float64)
        self._check(self.lib.gbfk_uq_dump(self.ctx, int(n), _ptr(out)))
        return out

    def set_observations(self, t1c, flair, pet=None, roi=None):
        t1 = np.ascontiguousarray(t1c, dtype=np.float64)
        fl = np.ascontiguousarray(flair, dtype=np.float64)
        pe = None if pet is None else np.ascontiguousarray(pet, dtype=np.float64)
        ro = None if roi is None else np.ascontiguousarray(roi, dtype=np.int32).reshape(-1, 3)
        self._check(self.lib.gbfk_set_observations(
            self.ctx, t1.shape[0], _ptr(t1), _ptr(fl), None if pe is None else _ptr(pe),
            None if ro is None else _ptr(ro), 0 if ro is None else ro.shape[0]))

    def log_likelihood(self, pet_sigma2=0.000361, pet_scale=0.85, t1_uc=0.7, t2_uc=0.25, slope=2.0, step_pet=1,
                       step_mri=1) -> np.ndarray:
        """[L_PET, L_T1c, L_FLAIR, sum] of the current phi (HGG_Likelihood::run)."""
        p = _lib.LikelihoodParams(pet_sigma2, pet_scale, t1_uc, t2_uc, slope, step_pet, step_mri)
        out = np.empty(4, dtype=np.float64)
        self._check(self.lib.gbfk_log_likelihood(self.ctx, ctypes.byref(p), _ptr(out)))
        return out


    # -- discrete adjoint ---------------------------------------------------
    def forward_adjoint(self, Dw, Dg, rho, dt, nsteps, x0=(0.0, 0.0, 0.0), sigma=0.0, nsnapshots=64, t1_uc=0.7,
                        t2_uc=0.25, slope=2.0, grad_c0=False, term_magnitudes=False):
        """Loss -(L_T1c + L_FLAIR) at the horizon and its gradients (gbfk_forward_adjoint).
        Returns a dict; with grad_c0 the dense d loss / d c0 is included, with
        term_magnitudes the sums of the magnitudes of the dDw and drho terms
        ("dDw_abs", "drho_abs")."""
        p = _lib.AdjointParams(float(Dw), float(Dg), float(rho), float(dt), int(nsteps), int(nsnapshots),
                               (ctypes.c_double * 3)(*[float(v) for v in x0]), float(sigma), float(t1_uc),
                               float(t2_uc), float(slope), _lib.ADJ_TERM_MAGNITUDES if term_magnitudes else 0)
        r = _lib.AdjointResult()
        g = np.empty((self.n, self.n, self.n), dtype=self.dtype) if grad_c0 else None
        self._check(self.lib.gbfk_forward_adjoint(self.ctx, ctypes.byref(p), ctypes.byref(r),
                                                  None if g is None else _ptr(g)))
        out = {"loss": r.loss, "dDw": r.dDw, "drho": r.drho, "dx0": np.array(list(r.dx0)),
               "forward_steps": int(r.forward_steps), "adjoint_steps": int(r.adjoint_steps)}
        if term_magnitudes:
            out["dDw_abs"], out["drho_abs"] = r.dDw_abs, r.drho_abs
        if g is not None:
            out["grad_c0"] = g
        return out


# ---------------------------------------------------------------- operators
class ReactionDiffusionOperator:
    """Tag for ReactionDiffusionOperator<3> (ReactionDiffusionOperator.h:21-43):
    coefficients in Real, stencil [-1, 2) in every direction."""

    stencil_start = (-1, -1, -1)
    stencil_end = (2, 2, 2)

    def __init__(self, Dw, Dg, rho):
        self.Dw, self.Dg, self.rho = Dw, Dg, rho


class UpdateTumor:
    """Tag for UpdateTumor<3> (ReactionDiffusionOperator.h:188-197)."""

    def __init__(self, dt):
        self.dt = float(dt)


class BlockProcessing:
    """Mirror of BlockProcessing_Pipeline_TBB's two entry points
    (MRAG/MRAGmultithreading/MRAGBlockProcessing_TBB.h:447-512) for the RD
    path.  ``vInfo`` and ``boundaryInfo`` are accepted for signature parity;
    the topology lives in the pool."""

    def __init__(self):
        self._pending = None

    def pipeline_process(self, vInfo, collection: BlockPool, boundaryInfo, op):
        if not isinstance(op, ReactionDiffusionOperator):
            raise TypeError("only ReactionDiffusionOperator runs on the device pool")
        self._pending = (collection, op)

    def process(self, vInfo, collection: BlockPool, op, granularity: int = -1):
        if not isinstance(op, UpdateTumor):
            raise TypeError("only UpdateTumor runs on the device pool")
        if self._pending is None or self._pending[0] is not collection:
            raise GbfkError(6, "UpdateTumor without a preceding ReactionDiffusionOperator sweep")
        _, rhs = self._pending
        self._pending = None
        collection.rd_step(rhs.Dw, rhs.Dg, rhs.rho, op.dt, 1)


def reaction_diffusion_step(pool: BlockPool, Dw, Dg, rho, dt, block_processing: BlockProcessing = None):
    """``Glioma_ReactionDiffusion::_reactionDiffusionStep`` on a device pool."""
    bp = block_processing or BlockProcessing()
    rhs = ReactionDiffusionOperator(Dw, Dg, rho)
    update = UpdateTumor(dt)
    bp.pipeline_process(None, pool, None, rhs)
    bp.process(None, pool, update, 4)
