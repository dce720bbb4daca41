"""Discrete adjoint of the fused step with binomial checkpointing
(gbfk_forward_adjoint): gradients of loss = -(L_T1c + L_FLAIR) w.r.t. Dw,
rho, the tumour origin x0 and the initial field, checked against central
finite differences (relative step 1e-4) of the same discrete forward map,
against finite differences of the oracle's forward run, across checkpoint
counts and across precisions."""
import numpy as np
import pytest

from gliomasolver_b200.anatomy import make_anatomy, tumor_ic
from gliomasolver_b200.schedule import make_schedule
from oracle import oracle as O

pytestmark = pytest.mark.gpu

N, BPD, L = 32, 4, 25.6
NSTEPS = 60
UC = dict(t1_uc=0.7, t2_uc=0.25, slope=2.0)


def _setup(prec, seed=0):
    from gliomasolver_b200 import BlockPool

    R = np.float64 if prec == "f64" else np.float32
    pw, pg, _ = make_anatomy(N, seed)
    sched = make_schedule(0.2, 0.1, 100.0, L, BPD, prec)
    pool = BlockPool(BPD ** 3, prec)
    pool.set_uniform(BPD)
    pool.upload_dense("p_w", pw.astype(R))
    pool.upload_dense("p_g", pg.astype(R))
    # synthetic observations: a ground-truth run thresholded at 0.7 / 0.25
    # with 2% of the labels flipped (seeded)
    x0_gt = (0.5, 0.45, 0.5)
    pool.upload_dense("phi", tumor_ic(N, x0_gt, pw, pg).astype(R))
    pool.rd_step(sched.Dw, sched.Dg, sched.rho, sched.dt, NSTEPS)
    u = pool.download_dense("phi").astype(np.float64)
    rng = np.random.default_rng(seed + 1)
    t1 = (u > 0.7).astype(float)
    fl = (u > 0.25).astype(float)
    for m in (t1, fl):
        flip = rng.random(m.shape) < 0.02
        m[flip] = 1 - m[flip]
    pool.set_observations(t1, fl)
    return pool, pw, pg, sched, t1, fl, R


def _coeffs(R, Dw_phys):
    Lr = R(L)
    Dw = R(R(Dw_phys) / (Lr * Lr))
    return float(Dw), float(R(0.1 * np.float64(Dw)))


def test_gradients_match_central_differences():
    pool, pw, pg, sched, t1, fl, R = _setup("f64")
    x0 = np.array([0.53, 0.47, 0.52])
    sigma = 2.0 / N
    Dw_phys, rho = 0.17, 0.08

    def run(dw, rh, xx):
        Dw, Dg = _coeffs(R, dw)
        return pool.forward_adjoint(Dw, Dg, rh, sched.dt, NSTEPS, x0=xx, sigma=sigma, nsnapshots=8, **UC)

    base = run(Dw_phys, rho, x0)
    assert base["adjoint_steps"] == NSTEPS
    # Dw (physical): d/dDw_phys = d/dDw_rescaled / L^2
    e = 1e-4 * Dw_phys
    fd = (run(Dw_phys + e, rho, x0)["loss"] - run(Dw_phys - e, rho, x0)["loss"]) / (2 * e)
    assert base["dDw"] / L ** 2 == pytest.approx(fd, rel=1e-5)
    e = 1e-4 * rho
    fd = (run(Dw_phys, rho + e, x0)["loss"] - run(Dw_phys, rho - e, x0)["loss"]) / (2 * e)
    assert base["drho"] == pytest.approx(fd, rel=1e-5)
    # The reference's Bernoulli term is discontinuous where u crosses uc
    # (omega2 = 1 for u > uc but (u-uc)^2 below, HGG_Likelihood.cpp:151-152):
    # moving the origin shifts the whole tumour, so a 1e-4 step pushes some
    # voxels across a threshold.  A 1e-7 step crosses none (FP64 forward).
    for d in range(3):
        e = 1e-7 * x0[d]
        xp, xm = x0.copy(), x0.copy()
        xp[d] += e
        xm[d] -= e
        fd = (run(Dw_phys, rho, xp)["loss"] - run(Dw_phys, rho, xm)["loss"]) / (2 * e)
        assert base["dx0"][d] == pytest.approx(fd, rel=1e-4, abs=1e-4)
    pool.close()


def test_initial_field_gradient_and_oracle_forward_differences():
    """d loss / d c0 along a random direction, and d loss / d Dw against
    central differences of the oracle's own forward solve + likelihood."""
    pool, pw, pg, sched, t1, fl, R = _setup("f64", seed=2)
    c0 = tumor_ic(N, (0.52, 0.5, 0.47), pw, pg)
    Dw, Dg = _coeffs(R, 0.15)
    rho = 0.06
    pool.upload_dense("phi", c0)
    res = pool.forward_adjoint(Dw, Dg, rho, sched.dt, NSTEPS, sigma=0.0, nsnapshots=5, grad_c0=True, **UC)
    g = res["grad_c0"]
    v = np.random.default_rng(3).standard_normal(c0.shape) * (c0 > 1e-3)
    eps = 1e-4

    def loss_from(c):
        pool.upload_dense("phi", c)
        return pool.forward_adjoint(Dw, Dg, rho, sched.dt, NSTEPS, sigma=0.0, nsnapshots=5, **UC)["loss"]

    fd = (loss_from(c0 + eps * v) - loss_from(c0 - eps * v)) / (2 * eps)
    assert np.sum(g * v) == pytest.approx(fd, rel=1e-5)

    # the oracle's forward map (C restatement of the reference, FP64)
    def oracle_loss(dw):
        d = np.float64(dw)
        u = O.rd_steps_dense(pw, pg, c0, d, np.float64(0.1 * d), rho, 1.0 / N, sched.dt, NSTEPS)
        lik = O.log_likelihood(u, t1, fl, None, **UC)
        return -(lik[1] + lik[2])

    e = 1e-4 * Dw
    fd = (oracle_loss(Dw + e) - oracle_loss(Dw - e)) / (2 * e)
    assert res["dDw"] == pytest.approx(fd, rel=1e-5)
    assert res["loss"] == pytest.approx(oracle_loss(Dw), rel=1e-12)
    pool.close()


def test_checkpoint_count_changes_cost_not_result():
    pool, pw, pg, sched, t1, fl, R = _setup("f64", seed=4)
    Dw, Dg = _coeffs(R, 0.2)
    out = [pool.forward_adjoint(Dw, Dg, 0.1, sched.dt, NSTEPS, x0=(0.5, 0.45, 0.5), sigma=2.0 / N,
                                nsnapshots=k, grad_c0=True, **UC) for k in (1, 3, 64)]
    for o in out[1:]:
        assert o["dDw"] == out[0]["dDw"] and o["drho"] == out[0]["drho"]
        assert np.array_equal(o["dx0"], out[0]["dx0"]) and np.array_equal(o["grad_c0"], out[0]["grad_c0"])
    steps = [o["forward_steps"] for o in out]
    assert steps[0] > steps[1] > steps[2] >= 2 * NSTEPS - 1
    pool.close()


def test_fp32_state_against_fp64():
    res = {}
    for prec in ("f64", "f32"):
        pool, pw, pg, sched, t1, fl, R = _setup(prec, seed=5)
        Dw, Dg = _coeffs(R, 0.18)
        res[prec] = pool.forward_adjoint(Dw, Dg, 0.07, make_schedule(0.2, 0.1, 100.0, L, BPD, "f64").dt, NSTEPS,
                                         x0=(0.5, 0.5, 0.5), sigma=2.0 / N, nsnapshots=8, **UC)
        pool.close()
    for k in ("loss", "dDw", "drho"):
        assert res["f32"][k] == pytest.approx(res["f64"][k], rel=2e-3), k
    assert np.allclose(res["f32"]["dx0"], res["f64"]["dx0"], rtol=2e-3, atol=1e-3 * np.abs(res["f64"]["dx0"]).max())


def test_autograd_function():
    import torch

    from gliomasolver_b200.autograd import tumor_loss

    pool, pw, pg, sched, t1, fl, R = _setup("f64", seed=6)
    Dw = torch.tensor(0.16, dtype=torch.float64, requires_grad=True)
    rho = torch.tensor(0.09, dtype=torch.float64, requires_grad=True)
    x0 = torch.tensor([0.5, 0.46, 0.5], dtype=torch.float64, requires_grad=True)
    loss = tumor_loss(pool, Dw, rho, x0, L, sched.dt, NSTEPS, 2.0 / N)
    loss.backward()
    Dwr, Dgr = _coeffs(R, 0.16)
    ref = pool.forward_adjoint(Dwr, Dgr, 0.09, sched.dt, NSTEPS, x0=(0.5, 0.46, 0.5), sigma=2.0 / N, **UC)
    assert float(loss) == ref["loss"]
    assert float(Dw.grad) == pytest.approx(ref["dDw"] / L ** 2, rel=1e-14)
    assert float(rho.grad) == ref["drho"]
    assert np.allclose(x0.grad.numpy(), ref["dx0"], rtol=1e-14)
    pool.close()
