"""Central-difference check of the discrete adjoint on a uniform grid.

``gbfk_forward_adjoint`` returns d loss / d Dw (Dg = 0.1 Dw), d loss / d rho
and d loss / d x0 for loss = -(L_T1c + L_FLAIR) of the state at the horizon
(HGG_Likelihood.cpp:136-156).  ``check_gradients`` compares them with central
differences of the forward map itself: plain forward solves on the same pool
(``gbfk_rd_step``, whose FP64 steps equal the reference's operator sweep bit
for bit) followed by the device likelihood.  The Bernoulli likelihood is
discontinuous where a voxel crosses a threshold (``omega2 = 1`` above ``uc``
but ``(u - uc)^2`` below, HGG_Likelihood.cpp:151-152), so a difference
quotient is only meaningful when no voxel crosses between the two runs;
``check_gradients`` counts the voxels that do and reports them beside each
quotient.
"""
from __future__ import annotations

import numpy as np

from .solver import BlockPool


def gaussian_ic(n: int, x0, sigma: float, p_w: np.ndarray, p_g: np.ndarray) -> np.ndarray:
    """The Gaussian initial condition of ``gbfk_forward_adjoint`` (sigma > 0):
    ``exp(-|x - x0|^2 / (2 sigma^2))`` at the vertex positions ``i / n`` where
    ``p_w + p_g > 0``, with ``|x - x0|^2`` summed over x, y, z in that order."""
    x = np.arange(n, dtype=np.float64) / n
    zz, yy, xx = np.meshgrid(x, x, x, indexing="ij")
    r2 = (xx - x0[0]) * (xx - x0[0]) + (yy - x0[1]) * (yy - x0[1]) + (zz - x0[2]) * (zz - x0[2])
    return np.where(p_w + p_g > 0, np.exp(-r2 / (2.0 * sigma * sigma)), 0.0)


def _forward(pool: BlockPool, c0, Dw, rho, dt, nsteps, uc):
    R = pool.dtype
    pool.upload_dense("phi", np.ascontiguousarray(c0, dtype=R))
    pool.rd_step(Dw, float(R(0.1 * np.float64(Dw))), rho, dt, nsteps)
    lik = pool.log_likelihood(t1_uc=uc[0], t2_uc=uc[1], slope=uc[2])
    return -(lik[1] + lik[2]), pool.download_dense("phi").astype(np.float64)


def _crossings(a: np.ndarray, b: np.ndarray, uc) -> int:
    return int(sum(np.count_nonzero((a > u) != (b > u)) for u in uc[:2]))


def check_gradients(pool: BlockPool, p_w, p_g, Dw, rho, dt, nsteps, x0, sigma, nsnapshots=64, rel_step=1e-4,
                    x_step=1e-7, t1_uc=0.7, t2_uc=0.25, slope=2.0) -> dict:
    """Adjoint gradients at (Dw, rho, x0) against central differences.

    ``pool`` holds the uniform grid with p_w, p_g and the observations
    (``set_observations``); ``p_w``, ``p_g`` are the same dense volumes (for
    the tissue mask of the initial condition).  Dw and Dw's step are in the
    rescaled units of ``gbfk_rd_step``; Dw and rho are perturbed by
    ``rel_step`` relative, each x0 component by ``x_step`` relative.  Returns
    the adjoint values, the difference quotients, their relative errors, the
    threshold crossings between each pair of runs and each quotient's
    resolution (one unit in the last place of the loss over the step, relative
    to the quotient), and dL/dx0 by the chain rule through the adjoint state
    at t = 0."""
    uc = (t1_uc, t2_uc, slope)
    R = pool.dtype
    Dg = float(R(0.1 * np.float64(Dw)))
    adj = pool.forward_adjoint(Dw, Dg, rho, dt, nsteps, x0=x0, sigma=sigma, nsnapshots=nsnapshots, t1_uc=t1_uc,
                               t2_uc=t2_uc, slope=slope, grad_c0=True, term_magnitudes=True)
    n = pool.n
    c0 = gaussian_ic(n, x0, sigma, p_w, p_g)
    out = {"loss": adj["loss"], "adjoint": {"dDw": adj["dDw"], "drho": adj["drho"], "dx0": list(adj["dx0"])},
           "forward_steps": adj["forward_steps"], "fd": {}, "rel_err": {}, "crossings": {},
           # sum of |term| over |sum of terms|: how much a relative change of the
           # terms (FP32 states) can move each gradient, relatively
           "term_cancellation": {"dDw": adj["dDw_abs"] / max(abs(adj["dDw"]), 1e-300),
                                 "drho": adj["drho_abs"] / max(abs(adj["drho"]), 1e-300)}}
    # dL/dx0 = sum_i dL/dc0_i * dc0_i/dx0 with dc0/dx0_d = c0 (x_d - x0_d) / sigma^2: the origin
    # gradient against the adjoint state at t = 0
    x = np.arange(n, dtype=np.float64) / n
    lam0 = adj["grad_c0"].astype(np.float64)
    w = lam0 * c0 / (sigma * sigma)
    chain = [float(np.sum(w * (x[None, None, :] - x0[0]))), float(np.sum(w * (x[None, :, None] - x0[1]))),
             float(np.sum(w * (x[:, None, None] - x0[2])))]
    out["chain_rule_dx0"] = chain
    out["chain_rule_rel_err"] = float(np.max(np.abs(np.array(adj["dx0"]) - chain)) / max(np.max(np.abs(chain)), 1e-300))
    # a difference quotient cannot resolve more than the rounding of the two
    # losses it subtracts: about one unit in the last place of each
    out["fd_resolution"] = {}

    def quotient(name, plus, minus, e, want):
        (lp, up), (lm, um) = plus, minus
        fd = (lp - lm) / (2 * e)
        out["fd"][name] = fd
        out["rel_err"][name] = abs(want - fd) / max(abs(fd), 1e-300)
        out["crossings"][name] = _crossings(up, um, uc)
        out["fd_resolution"][name] = float(np.spacing(max(abs(lp), abs(lm))) / (2 * e) / max(abs(fd), 1e-300))

    e = rel_step * Dw
    quotient("dDw", _forward(pool, c0, Dw + e, rho, dt, nsteps, uc), _forward(pool, c0, Dw - e, rho, dt, nsteps, uc),
             e, adj["dDw"])
    e = rel_step * rho
    quotient("drho", _forward(pool, c0, Dw, rho + e, dt, nsteps, uc), _forward(pool, c0, Dw, rho - e, dt, nsteps, uc),
             e, adj["drho"])
    for d in range(3):
        e = x_step * x0[d]
        xp, xm = list(x0), list(x0)
        xp[d] += e
        xm[d] -= e
        quotient(f"dx0[{d}]", _forward(pool, gaussian_ic(n, xp, sigma, p_w, p_g), Dw, rho, dt, nsteps, uc),
                 _forward(pool, gaussian_ic(n, xm, sigma, p_w, p_g), Dw, rho, dt, nsteps, uc), e, adj["dx0"][d])
    return out


def synthetic_observations(pool: BlockPool, c0, Dw, rho, dt, nsteps, seed, t1_uc=0.7, t2_uc=0.25, flip=0.02):
    """Observed masks of a calibration problem: a ground-truth forward run on
    ``pool`` from ``c0``, thresholded at ``t1_uc`` (enhancing core, T1c) and
    ``t2_uc`` (edema, FLAIR) as Glioma_UQ_DataPreprocessing.cpp:194-232 does,
    with a seeded fraction ``flip`` of the labels flipped; set as the pool's
    observations and returned."""
    R = pool.dtype
    pool.upload_dense("phi", np.ascontiguousarray(c0, dtype=R))
    pool.rd_step(Dw, float(R(0.1 * np.float64(Dw))), rho, dt, nsteps)
    u = pool.download_dense("phi").astype(np.float64)
    rng = np.random.default_rng(seed)
    masks = [(u > t1_uc).astype(float), (u > t2_uc).astype(float)]
    for m in masks:
        f = rng.random(m.shape) < flip
        m[f] = 1 - m[f]
    pool.set_observations(*masks)
    return masks


def config5_sample(i, n=256, seed=5):
    """Sample i of the batched forward + adjoint workload (config 5): its own
    seeded anatomy (brain scale U[0.8, 1.2]) and parameters drawn as for a
    TMCMC stage (Dw log-U[0.02, 0.3] cm^2/day, rho log-U[0.002, 0.2] / day,
    T U[30, 300] d, x0 a white-matter voxel).  Returns (p_w, p_g, sample,
    rng), rng seeded for the sample (its label noise)."""
    from .anatomy import make_anatomy
    from .tmcmc import sample_stage

    rng = np.random.default_rng([seed, i])
    p_w, p_g, _ = make_anatomy(n, seed + 100 + i, scale=float(rng.uniform(0.8, 1.2)))
    st = sample_stage(1, p_w, seed=seed + 200 + i)[0]
    return p_w, p_g, st, rng
