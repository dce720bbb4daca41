"""Batched evaluation of a TMCMC stage's forward solves.

In the reference a TMCMC stage (tools/pi4u_lite/Inference/engine_tmcmc.c:
597-624) runs one solver process per parameter sample: fitfun_glioma.c:46-245
writes InputParameters.txt (Dw, rho, Tend) and TumorIC.txt (x0), forks
runAll.sh, which runs ``brain -model RD -UQ 1`` and the likelihood.  Here a
``Batch`` holds every sample of a stage on the GPU and advances them together
(gbfk_batch_* in include/gbfk.h); each sample keeps the reference's own
schedule (its dt from its own Dw, its own step count to its own Tend,
Glioma_ReactionDiffusion.cpp:300-321).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import GbfkError
from .schedule import make_schedule


@dataclass
class StageSample:
    Dw_cm2_day: float
    rho_day: float
    tend_day: float
    x0: tuple


def sample_stage(nsamples: int, p_w: np.ndarray, seed: int = 0, Dw_range=(0.02, 0.3), rho_range=(0.002, 0.2),
                 tend_range=(30.0, 300.0)):
    """Seeded stage parameters: Dw and rho log-uniform, Tend uniform, x0 a
    uniformly chosen white-matter voxel (P_WM > 0.5)."""
    rng = np.random.default_rng(seed)
    n = p_w.shape[0]
    Dw = np.exp(rng.uniform(np.log(Dw_range[0]), np.log(Dw_range[1]), nsamples))
    rho = np.exp(rng.uniform(np.log(rho_range[0]), np.log(rho_range[1]), nsamples))
    tend = rng.uniform(tend_range[0], tend_range[1], nsamples)
    cand = np.flatnonzero(p_w.ravel() > 0.5)
    idx = cand[rng.integers(0, cand.size, nsamples)]
    iz, iy, ix = np.unravel_index(idx, p_w.shape)
    return [StageSample(float(Dw[i]), float(rho[i]), float(tend[i]), (ix[i] / n, iy[i] / n, iz[i] / n))
            for i in range(nsamples)]


def to_gbfk_samples(stage, blocks_per_dim: int, precision: str, L_cm: float = 25.6, anatomy=None):
    """Per-sample schedules in the build's Real, as gbfk_sample records."""
    n = 8 * blocks_per_dim
    out = (_lib.Sample * len(stage))()
    scheds = []
    for i, s in enumerate(stage):
        sch = make_schedule(s.Dw_cm2_day, s.rho_day, s.tend_day, L_cm, blocks_per_dim, precision)
        scheds.append(sch)
        r = out[i]
        r.Dw, r.Dg, r.rho, r.dt, r.nsteps = sch.Dw, sch.Dg, sch.rho, sch.dt, sch.nsteps
        r.anatomy = 0 if anatomy is None else int(anatomy[i])
        r.x0[0], r.x0[1], r.x0[2] = s.x0
        r.sigma = 2.0 / n
    return out, scheds


class Batch:
    """A gbfk_batch: all forward solves of a stage on one GPU."""

    def __init__(self, blocks_per_dim: int, max_samples: int, precision: str = "f32", max_anatomies: int = 1,
                 device: int = 0, stream=None):
        self.lib = _lib.load()
        self.precision = precision
        self.dtype = np.float64 if precision == "f64" else np.float32
        self.n = 8 * blocks_per_dim
        cfg = _lib.Config(_lib.GBFK_F64 if precision == "f64" else _lib.GBFK_F32, 1, int(device), stream)
        h = ctypes.c_void_p()
        rc = self.lib.gbfk_batch_create(ctypes.byref(cfg), int(blocks_per_dim), int(max_samples),
                                        int(max_anatomies), ctypes.byref(h))
        if rc != _lib.GBFK_OK:
            raise GbfkError(rc, "gbfk_batch_create failed")
        self.b = h
        self._samples = None

    def _check(self, rc):
        if rc != _lib.GBFK_OK:
            msg = self.lib.gbfk_batch_last_error(self.b)
            raise GbfkError(rc, msg.decode() if msg else "")

    def close(self):
        if getattr(self, "b", None):
            self.lib.gbfk_batch_destroy(self.b)
            self.b = None

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
        return int(self.lib.gbfk_batch_launch_count(self.b))

    @property
    def samples_per_cta(self) -> int:
        return int(self.lib.gbfk_batch_samples_per_cta(self.b))

    def set_anatomy(self, index: int, p_w: np.ndarray, p_g: np.ndarray):
        a = np.ascontiguousarray(p_w, dtype=self.dtype)
        g = np.ascontiguousarray(p_g, dtype=self.dtype)
        self._check(self.lib.gbfk_batch_set_anatomy(self.b, int(index), a.ctypes.data_as(ctypes.c_void_p),
                                                    g.ctypes.data_as(ctypes.c_void_p)))

    def set_samples(self, samples):
        self._samples = samples  # keep the ctypes array alive
        self._check(self.lib.gbfk_batch_set_samples(self.b, len(samples), samples))

    def run(self, samples_per_cta: int = 0):
        """Run every sample to its horizon: samples_per_cta -1 = the
        pipelined step, 1/2/4 = the per-block kernel, 0 = autotune."""
        self._check(self.lib.gbfk_batch_run(self.b, int(samples_per_cta)))

    def set_observations(self, t1c, flair, pet=None, roi=None):
        """Observations of the likelihood step on the batch's n^3 grid (as
        BlockPool.set_observations), shared by every sample."""
        t1 = np.ascontiguousarray(t1c, dtype=np.float64)
        fl = np.ascontiguousarray(flair, dtype=np.float64)
        pe = None if pet is None else np.ascontiguousarray(pet, dtype=np.float64)
        ro = None if roi is None else np.ascontiguousarray(roi, dtype=np.int32).reshape(-1, 3)
        self._keep_obs = (t1, fl, pe, ro)
        ptr = lambda a: None if a is None else a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
        self._check(self.lib.gbfk_batch_set_observations(self.b, ptr(t1), ptr(fl), ptr(pe), ptr(ro),
                                                         0 if ro is None else ro.shape[0]))

    def log_likelihood(self, pet_sigma2=0.000361, pet_scale=0.85, t1_uc=0.7, t2_uc=0.25, slope=2.0, step_pet=1,
                       step_mri=1) -> np.ndarray:
        """[L_PET, L_T1c, L_FLAIR, sum] of every sample after run(), shape
        (samples, 4), in the order of set_samples (HGG_Likelihood::run)."""
        p = _lib.LikelihoodParams(pet_sigma2, pet_scale, t1_uc, t2_uc, slope, step_pet, step_mri)
        n = len(self._samples) if self._samples is not None else 0
        out = np.empty((n, 4), dtype=np.float64)
        self._check(self.lib.gbfk_batch_log_likelihood(self.b, ctypes.byref(p), out.ctypes.data_as(ctypes.c_void_p)))
        return out

    def download(self, sample: int) -> np.ndarray:
        out = np.empty((self.n, self.n, self.n), dtype=self.dtype)
        self._check(self.lib.gbfk_batch_download(self.b, int(sample), out.ctypes.data_as(ctypes.c_void_p)))
        return out
