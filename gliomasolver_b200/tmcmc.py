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
from dataclasses import dataclass, field

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


def to_gbfk_samples(stage, blocks_per_dim: int, precision: str, L_cm: float = 25.6, anatomy=None, ic="gaussian"):
    """Per-sample schedules in the build's Real, as gbfk_sample records.
    ``ic``: "gaussian" (c0 = exp(-|x-x0|^2 / (2 (2h)^2)), the synthetic
    workloads' initial condition) or "ball" (the reference's smoothed-ball
    tumour of Glioma_ReactionDiffusion::_ic)."""
    kind = _lib.IC_KINDS[ic]
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
        r.ic = kind
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

    @property
    def tile_shape(self) -> tuple:
        """(consumer warps, heavy slots, empty slots) of the pipelined step the
        last run used; (0, 0, 0) for the per-block kernel."""
        sh = (ctypes.c_int * 3)()
        self._check(self.lib.gbfk_batch_tile_shape(self.b, ctypes.byref(sh)))
        return tuple(sh)

    @property
    def graph_count(self) -> int:
        """CUDA graphs the last run replayed."""
        return int(self.lib.gbfk_batch_graph_count(self.b))

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
        (samples, 4), in the order of set_samples (HGG_Likelihood::run).
        pet_sigma2 .. slope may be scalars or one value per sample."""
        n = len(self._samples) if self._samples is not None else 0
        cols = [np.broadcast_to(np.asarray(v, dtype=np.float64), (n,)) for v in
                (pet_sigma2, pet_scale, t1_uc, t2_uc, slope)]
        per_sample = any(np.ndim(v) > 0 for v in (pet_sigma2, pet_scale, t1_uc, t2_uc, slope))
        m = n if per_sample else 1
        ps = (_lib.LikelihoodParams * max(m, 1))()
        for i in range(m):
            ps[i] = _lib.LikelihoodParams(*(float(c[i]) for c in cols), int(step_pet), int(step_mri))
        out = np.empty((n, 4), dtype=np.float64)
        self._check(self.lib.gbfk_batch_log_likelihood(self.b, ps, int(per_sample), out.ctypes.data_as(ctypes.c_void_p)))
        return out

    def download(self, sample: int) -> np.ndarray:
        out = np.empty((self.n, self.n, self.n), dtype=self.dtype)
        self._check(self.lib.gbfk_batch_download(self.b, int(sample), out.ctypes.data_as(ctypes.c_void_p)))
        return out


# ---------------------------------------------------------------------------
# In-process TMCMC (transitional Markov chain Monte Carlo).
#
# The reference's engine (tools/pi4u_lite/Inference/engine_tmcmc.c with
# tmcmc_stats.c) tempers the likelihood, L^p_j with p_0 = 0 .. 1, stage by
# stage.  Per stage: the next exponent makes the coefficient of variation of
# the plausibility weights L^(p_{j+1} - p_j) equal TolCOV
# (calculate_statistics, tmcmc_stats.c:545-620); the stage's log-evidence
# factor is log(sum w) + max - log n (:641-652); PopSize leaders are drawn
# multinomially by weight; the proposal covariance is bbeta times the
# weighted sample covariance (:700-757, compute_candidate engine_tmcmc.c:
# 661-681, redrawn until inside the bounds); chains longer than
# MaxChainLength are split (prepare_newgen :880-900); each chain step is a
# Metropolis decision at p_{j+1} with a uniform prior (chaintask :683-738).
# Here every chain's step k of a stage is evaluated in one call of the
# log-likelihood over all proposals (one batched launch for the glioma model)
# instead of one solver process per sample.

@dataclass
class TMCMCOptions:
    pop_size: int = 512
    max_stages: int = 100         # MaxStages: generations, the prior one included
    tol_cov: float = 1.0          # TolCOV
    opt_tol: float = 1e-6         # opt.Tol: fzerofind's acceptance of |objlogp| (engine_tmcmc.c:75)
    bbeta: float = 0.2            # proposal covariance scale
    min_chain: int = 0            # MinChainLength
    max_chain: int = 1            # MaxChainLength
    seed: int = 280675
    penalty: float = -1.0e12      # log-likelihood of a failed / NaN evaluation (fitfun_glioma.c:203-217)


@dataclass
class TMCMCResult:
    theta: np.ndarray             # final population (pop_size, d)
    loglik: np.ndarray            # its log-likelihoods
    p: list                       # tempering exponents p_0 = 0 .. p_last
    log_evidence: float
    acceptance: list              # per stage: accepted proposals / proposals
    evaluations: int
    # Per generation g = 0 .. len(p) - 1, the quantities the reference keeps
    # in its run record (engine_tmcmc.c:334-365, tmcmc_stats.c
    # calculate_statistics): the population and its log-likelihoods, the
    # distinct points among them, the COV of the weights that lead to
    # generation g + 1, log of the evidence increment, the weighted mean and
    # the weighted (unscaled) sample covariance.
    stages: list = field(default_factory=list)          # [(theta, F)]
    uniques: list = field(default_factory=list)
    coef_var: list = field(default_factory=list)
    log_selection: list = field(default_factory=list)
    mean_theta: list = field(default_factory=list)
    ss: np.ndarray = None                                # of the last generation
    p_next: float = None                                 # exponent after the last generation (set at the end)


@dataclass
class TMCMCCheckpoint:
    """A run stopped after generation G = len(result.stages) - 1, with the
    random generator's state at that point (``tmcmc(..., start=...)``)."""
    result: TMCMCResult
    rng_state: dict


FZERO_STEP = 1e-4  # the exponent grid of fzerofind (tmcmc_stats.c:104)
_FZERO_CHUNK = 2048


def _seqsum(a, axis=-1):
    """Sum in index order, as the reference's loops add (numpy's own sum is
    pairwise and rounds differently)."""
    return np.cumsum(a, axis=axis).take(-1, axis=axis)


def objlogp(x, F, pj, tol_cov):
    """(COV of the weights exp((F - max F) (x - pj)) - tol_cov)^2 for each
    exponent in ``x`` (Objlogp, tmcmc_stats.c:18-50: weights normalised by
    their sum, mean and sample standard deviation, sums in index order)."""
    x = np.atleast_1d(np.asarray(x, dtype=np.float64))
    F = np.asarray(F, dtype=np.float64)
    n = F.size
    with np.errstate(over="ignore", invalid="ignore", divide="ignore"):
        w = np.exp((F - F.max())[None, :] * (x - pj)[:, None])
        q = w / _seqsum(w)[:, None]
        mean = _seqsum(q) / n
        std = np.sqrt(_seqsum((q - mean[:, None]) ** 2) / (n - 1))
        return (std / mean - tol_cov) ** 2


def fzerofind(F, pj, tol_cov, opt_tol):
    """The reference's exponent search (fzerofind, tmcmc_stats.c:96-215):
    objlogp on the grid x = x_lo + k step of [0, 4) with step 1e-4, in order,
    keeping the first smallest value and stopping at the first value within
    opt_tol; without such a value the grid is refined around the smallest one
    (+-10 steps, step / 10) until the step falls below 1e-16.  Returns
    (converged, x, f); the reference returns "converged" with x = f = 0 when
    the step runs out."""
    x_lo, x_hi, step = 0.0, 4.0, FZERO_STEP
    while True:
        niters = int((x_hi - x_lo) / step)
        m, fm, found = 0.0, np.finfo(np.float64).max, False
        for start in range(0, niters, _FZERO_CHUNK):
            it = np.arange(start, min(niters, start + _FZERO_CHUNK), dtype=np.float64)
            xs = x_lo + it * step
            fx = objlogp(xs, F, pj, tol_cov)
            with np.errstate(invalid="ignore"):
                hit = np.flatnonzero(np.abs(fx) <= opt_tol)
            seg = fx[: hit[0] + 1] if hit.size else fx
            valid = np.flatnonzero(~np.isnan(seg))
            if valid.size:
                k = valid[np.argmin(seg[valid])]
                if seg[k] < fm:
                    fm, m = float(seg[k]), float(xs[k])
            if hit.size:
                found = True
                break
        if found:
            return True, m, fm
        x_lo = max(m - 10 * step, 0.0)
        x_hi = min(m + 10 * step, 4.0)
        step = 0.1 * step
        if step < 1e-16:
            return True, 0.0, 0.0


def force_pos_def(S):
    """Diagonal loading until S is positive definite (force_pos_def2,
    posdef.c:273-341): while an eigenvalue is not positive, add
    max(0.01 max|diag|, 1e-15) - min(diag, 0) to the diagonal if some
    diagonal entry is at most 1e-15, else scale the diagonal by 1.01."""
    S = np.array(S, dtype=np.float64, copy=True)
    while not np.all(np.linalg.eigvalsh(S) > 0):
        d = np.diag(S).copy()
        m = np.max(np.abs(d)) * 0.01
        if np.any(d <= 1e-15):
            neg = d.min()
            addit = m - neg if neg < 0 else max(m, 1e-15)
            S[np.diag_indices_from(S)] = d + addit
        else:
            S[np.diag_indices_from(S)] = d * 1.01
    return S


def make_posdef(S):
    """S unchanged when positive definite, else force_pos_def (make_posdef
    with method 2, posdef.c:577-616, as calculate_statistics calls it)."""
    S = np.asarray(S, dtype=np.float64)
    return S.copy() if np.all(np.linalg.eigvalsh(S) > 0) else force_pos_def(S)


@dataclass
class StageStatistics:
    p_next: float        # the next tempering exponent
    coef_var_next: float  # the search's objective there (CoefVar[gen + 1] until the next stage)
    coef_var: float      # COV of the weights toward p_next (CoefVar[gen])
    log_selection: float  # log evidence increment (logselection[gen])
    q: np.ndarray        # normalised weights
    mean: np.ndarray     # weighted mean of the population (meantheta[gen])
    ss: np.ndarray       # weighted sample covariance, made positive definite (SS)


def cov_root(F, pj, tol_cov, opt_tol):
    """The exponent search the reference tries first (fminsearch,
    tmcmc_stats.c:315-408: GSL's simplex minimiser of objlogp started at pj),
    here as bisection for COV = tol_cov on (pj, pj + 4] (the COV of the
    weights grows with the exponent above pj).  Returns (converged, x, f)
    with the reference's convergence test |f| <= opt_tol; without a root in
    the bracket it reports no convergence, as the simplex search does when
    the target COV is out of reach."""
    F = np.asarray(F, dtype=np.float64)
    lo, hi = pj, pj + 4.0
    if objlogp(hi, F, pj, tol_cov)[0] <= opt_tol:
        return True, hi, float(objlogp(hi, F, pj, tol_cov)[0])

    def cov(x):
        return np.sqrt(objlogp(x, F, pj, 0.0)[0])

    if not cov(hi) > tol_cov:
        return False, 0.0, 0.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if mid in (lo, hi):
            break
        if cov(mid) > tol_cov:
            hi = mid
        else:
            lo = mid
    x = hi if abs(cov(hi) - tol_cov) <= abs(cov(lo) - tol_cov) else lo
    f = float(objlogp(x, F, pj, tol_cov)[0])
    return (abs(f) <= opt_tol), x, f


def next_exponent_search(F, pj, tol_cov, opt_tol):
    """(p_next, objective there) as calculate_statistics sets them
    (tmcmc_stats.c:558-617): the root search, then fzerofind if it did not
    converge; the result if it lies above pj, else pj + 1e-5; at most 1."""
    conv, xmin, fmin = cov_root(F, pj, tol_cov, opt_tol)
    if not conv:
        conv, xmin, fmin = fzerofind(F, pj, tol_cov, opt_tol)
    if conv and xmin > pj:
        pn, fn = xmin, fmin
    else:
        pn, fn = pj + 0.1 * FZERO_STEP, float("nan")
    return min(pn, 1.0), fn


def stage_statistics(F, theta, pj, tol_cov, opt_tol, p_next=None):
    """calculate_statistics (tmcmc_stats.c:545-765) for one generation: the
    next exponent (next_exponent_search, or ``p_next`` when given); weights
    exp(F (p_next - pj) - max) normalised by their sum in index order; log
    evidence increment log(sum) + max - log(n); the weighted mean and
    covariance summed over the population in index order (the covariance
    entry (a, b) takes its product in the order (max(a, b), min(a, b)), the
    last one the reference writes), made positive definite."""
    F = np.asarray(F, dtype=np.float64)
    theta = np.asarray(theta, dtype=np.float64)
    n, d = theta.shape
    if p_next is None:
        pn, cvn = next_exponent_search(F, pj, tol_cov, opt_tol)
    else:
        pn, cvn = float(p_next), float("nan")
    flcp = F * (pn - pj)
    fjmax = flcp.max()
    w = np.exp(flcp - fjmax)
    sw = float(_seqsum(w))
    q = w / sw
    log_sel = float(np.log(sw) + fjmax - np.log(n))
    mq = float(_seqsum(q)) / n
    cv = float(np.sqrt(_seqsum((q - mq) ** 2) / (n - 1)) / mq)
    mean = _seqsum(theta * q[:, None], axis=0)
    dev = theta - mean
    ss = np.empty((d, d))
    for a in range(d):
        for b in range(d):
            hi, lo = max(a, b), min(a, b)
            ss[a, b] = _seqsum((q * dev[:, hi]) * dev[:, lo])
    return StageStatistics(float(pn), float(cvn), cv, log_sel, q, mean, make_posdef(ss))


def next_exponent(F, p, tol_cov, opt_tol=1e-6):
    """The exponent after p (next_exponent_search)."""
    return next_exponent_search(np.asarray(F, dtype=np.float64), p, tol_cov, opt_tol)[0]


def _distinct_points(theta, tol=1e-6):
    """How many points of the population differ from every earlier distinct
    one in some coordinate by more than tol (engine_tmcmc.c:795-835)."""
    table = np.empty_like(theta)
    un = 0
    for x in theta:
        if un == 0 or not np.any(np.all(np.abs(table[:un] - x) <= tol, axis=1)):
            table[un] = x
            un += 1
    return un


def tmcmc(loglik, lower, upper, opts: TMCMCOptions = TMCMCOptions(), on_generation=None, start=None):
    """Sample the posterior of a uniform prior on the box [lower, upper]
    times exp(loglik).  ``loglik(theta)`` takes an (n, d) array and returns n
    log-likelihoods (NaN/inf count as ``opts.penalty``).

    ``on_generation(result, rng_state)`` is called once per generation, after
    its statistics are recorded (``result.stages[-1]`` is its population,
    ``result.p[-1]`` its exponent; ``result.p_next`` is None until the last
    one), with the random generator's state at that point, which is the start
    of the generation's transition (``tmcmc_io.Checkpointer`` writes the
    reference's files and the exact state there).  ``start``: a
    ``TMCMCCheckpoint`` (``tmcmc_io.load_checkpoint``); the run continues
    from its last generation and, with the same likelihood and options,
    equals the uninterrupted run."""
    rng = np.random.default_rng(opts.seed)
    lower = np.asarray(lower, dtype=np.float64)
    upper = np.asarray(upper, dtype=np.float64)
    d = lower.size
    nevals = 0

    def evaluate(th):
        nonlocal nevals
        nevals += len(th)
        F = np.asarray(loglik(th), dtype=np.float64)
        return np.where(np.isfinite(F), F, opts.penalty)

    log_ev = 0.0
    if start is None:
        theta = lower + (upper - lower) * rng.random((opts.pop_size, d))
        F = evaluate(theta)
        p = [0.0]
        acc = []
        rec = TMCMCResult(None, None, p, 0.0, acc, 0)
    else:
        # generations 0..G-1 as recorded; G's statistics are recomputed below
        old = start.result
        g = len(old.stages) - 1
        theta, F = (a.copy() for a in old.stages[g])
        p, acc = list(old.p[:g + 1]), list(old.acceptance[:g])
        rec = TMCMCResult(None, None, p, 0.0, acc, 0, stages=list(old.stages[:g]), uniques=list(old.uniques[:g]),
                          coef_var=list(old.coef_var[:g]), log_selection=list(old.log_selection[:g]),
                          mean_theta=list(old.mean_theta[:g]))
        for v in rec.log_selection:
            log_ev += v
        nevals = old.evaluations
        rng.bit_generator.state = start.rng_state

    def record(theta, F, st):
        rec.stages.append((theta.copy(), F.copy()))
        rec.uniques.append(_distinct_points(theta))
        rec.coef_var.append(st.coef_var)
        rec.log_selection.append(st.log_selection)
        rec.mean_theta.append(st.mean)
        rec.ss = st.ss
        rec.theta, rec.loglik, rec.log_evidence, rec.evaluations = theta, F, float(log_ev), nevals
        if on_generation is not None:
            on_generation(rec, rng.bit_generator.state)

    done = p[-1] >= 1.0
    for _ in range(0 if done else opts.max_stages - len(p)):
        pj = p[-1]
        st = stage_statistics(F, theta, pj, opts.tol_cov, opts.opt_tol)
        pn, q = st.p_next, st.q
        log_ev += st.log_selection
        record(theta, F, st)
        sel = rng.multinomial(opts.pop_size, q)
        # the proposal covariance bbeta * SS (compute_candidate, engine_tmcmc.c:661-681)
        cov = opts.bbeta * st.ss
        # leaders with chain lengths (split at max_chain, raised to min_chain)
        chains = []
        for i in np.flatnonzero(sel):
            k = int(sel[i])
            while opts.max_chain > 0 and k > opts.max_chain:
                chains.append([i, opts.max_chain])
                k -= opts.max_chain
            chains.append([i, max(k, opts.min_chain)])
        lead = np.array([theta[i] for i, _ in chains])
        flead = np.array([F[i] for i, _ in chains])
        steps = np.array([k for _, k in chains])
        chol = np.linalg.cholesky(cov)
        new_theta, new_F = [], []
        naccept = nprop = 0
        for s in range(int(steps.max()) if len(steps) else 0):
            act = np.flatnonzero(steps > s)
            cand = np.empty((len(act), d))
            for j, c in enumerate(act):
                for _try in range(10000):
                    x = lead[c] + chol @ rng.standard_normal(d)
                    if np.all(x >= lower) and np.all(x <= upper):
                        break
                else:
                    x = np.clip(x, lower, upper)
                cand[j] = x
            fc = evaluate(cand)
            u = rng.random(len(act))
            ok = u < np.exp(np.minimum(0.0, (fc - flead[act]) * pn))
            naccept += int(ok.sum())
            nprop += len(act)
            lead[act[ok]] = cand[ok]
            flead[act[ok]] = fc[ok]
            new_theta.append(lead[act].copy())
            new_F.append(flead[act].copy())
        theta = np.concatenate(new_theta) if new_theta else theta
        F = np.concatenate(new_F) if new_F else F
        p.append(pn)
        acc.append(naccept / max(nprop, 1))
        if pn >= 1.0:
            break
    # The last generation's own statistics, toward the exponent that would
    # follow it (1 after the final stage, so uniform weights), as the
    # reference computes them after its last stage.
    st = stage_statistics(F, theta, p[-1], opts.tol_cov, opts.opt_tol)
    rec.p_next = st.p_next
    log_ev += st.log_selection
    record(theta, F, st)
    rec.theta, rec.loglik, rec.log_evidence, rec.evaluations = theta, F, float(log_ev), nevals
    return rec


class GliomaModel:
    """The likelihood of the reference's glioma calibration
    (fitfun_glioma.c:128-151) evaluated for a whole population at once:
    theta = log of (Dw [cm^2/day], rho [1/day], c = Tend^2 rho, x0, y0, z0,
    PET sigma, PET scale, T1c threshold, FLAIR threshold, sigmoid slope)
    rows; every row's forward solve runs in one batch and its likelihood on
    the device after it.  ``ic="ball"`` starts every row from the
    reference's smoothed-ball tumour at (x0, y0, z0), as its TumorIC.txt
    runs do (Glioma_ReactionDiffusion.cpp:39-52,155-164)."""

    def __init__(self, p_w, p_g, t1c, flair, pet=None, roi=None, L_cm=25.6, precision="f32", max_samples=4096,
                 device=0, stream=None, step_pet=1, step_mri=1, ic="gaussian"):
        n = p_w.shape[0]
        if n % 8:
            raise ValueError("the grid must be 8 * blocks per direction")
        self.bpd = n // 8
        self.n = n
        self.L_cm = L_cm
        self.precision = precision
        self.steps = (step_pet, step_mri)
        self.ic = ic
        self.batch = Batch(self.bpd, max_samples, precision, device=device, stream=stream)
        R = np.float64 if precision == "f64" else np.float32
        self.batch.set_anatomy(0, p_w.astype(R), p_g.astype(R))
        self.batch.set_observations(t1c, flair, pet, roi)
        self.max_samples = max_samples

    def parameters(self, theta):
        v = np.exp(np.asarray(theta, dtype=np.float64))
        Dw, rho = v[:, 0], v[:, 1]
        tend = np.sqrt(v[:, 2] / rho)
        return Dw, rho, tend, v[:, 3:6], v[:, 6] ** 2, v[:, 7], v[:, 8], v[:, 9], v[:, 10]

    def __call__(self, theta):
        Dw, rho, tend, x0, pet_s2, pet_scale, t1uc, t2uc, slope = self.parameters(theta)
        out = np.empty(len(Dw))
        for a in range(0, len(Dw), self.max_samples):
            sl = slice(a, min(a + self.max_samples, len(Dw)))
            stage = [StageSample(float(Dw[i]), float(rho[i]), float(tend[i]), tuple(x0[i])) for i in
                     range(sl.start, sl.stop)]
            samples, _ = to_gbfk_samples(stage, self.bpd, self.precision, self.L_cm, ic=self.ic)
            self.batch.set_samples(samples)
            try:
                self.batch.run(0)
            except GbfkError as e:
                if e.code != _lib.STATUS_CODES["GBFK_E_NAN"]:
                    raise
            lik = self.batch.log_likelihood(pet_s2[sl], pet_scale[sl], t1uc[sl], t2uc[sl], slope[sl], *self.steps)
            out[sl] = lik[:, 3]
        return out

    def close(self):
        self.batch.close()
