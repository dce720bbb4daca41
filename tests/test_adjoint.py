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
    # revolve's minimal counts for 60 steps (the first sweep to the horizon
    # included): 1 buffer 390, 3 buffers 188; with 64 buffers the first sweep
    # stores every state and nothing is recomputed
    assert steps == [390, 188, NSTEPS]
    pool.close()


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_forward_stream_of_its_own_gives_the_same_bits(prec, monkeypatch):
    """The reverse sweep's recomputation on a stream of its own (the default)
    and on the caller's stream (GBFK_ADJ_STREAMS=1) give the same bits, with
    few checkpoint buffers (much recomputation, buffers reused first-in
    first-out) and with every state kept."""
    pool, pw, pg, sched, t1, fl, R = _setup(prec, seed=6)
    Dw, Dg = _coeffs(R, 0.2)

    def run(k):
        return pool.forward_adjoint(Dw, Dg, 0.1, sched.dt, NSTEPS, x0=(0.5, 0.45, 0.5), sigma=2.0 / N,
                                    nsnapshots=k, grad_c0=True, **UC)

    for k in (2, 5, 64):
        monkeypatch.delenv("GBFK_ADJ_STREAMS", raising=False)
        two = run(k)
        monkeypatch.setenv("GBFK_ADJ_STREAMS", "1")
        one = run(k)
        assert two["forward_steps"] == one["forward_steps"]
        for key in ("loss", "dDw", "drho"):
            assert two[key] == one[key], (k, key)
        assert np.array_equal(two["dx0"], one["dx0"]) and np.array_equal(two["grad_c0"], one["grad_c0"])
    pool.close()


def test_fp32_state_against_fp64():
    """FP32 state against FP64 on the same problem.  A gradient is a sum of
    terms over cells and steps; a relative change e of the terms (the FP32
    state's rounding) moves it by up to e * sum|term|, so the bound is scaled
    by the cancellation sum|term| / |sum term| measured in FP64
    (GBFK_ADJ_TERM_MAGNITUDES)."""
    res = {}
    for prec in ("f64", "f32"):
        pool, pw, pg, sched, t1, fl, R = _setup(prec, seed=5)
        Dw, Dg = _coeffs(R, 0.18)
        res[prec] = pool.forward_adjoint(Dw, Dg, 0.07, make_schedule(0.2, 0.1, 100.0, L, BPD, "f64").dt, NSTEPS,
                                         x0=(0.5, 0.5, 0.5), sigma=2.0 / N, nsnapshots=8,
                                         term_magnitudes=prec == "f64", **UC)
        pool.close()
    a, b = res["f64"], res["f32"]
    cancel = {k: a[k + "_abs"] / abs(a[k]) for k in ("dDw", "drho")}
    rel = {k: abs(b[k] - a[k]) / abs(a[k]) for k in ("loss", "dDw", "drho")}
    print(cancel, rel)
    assert rel["loss"] <= 1e-5
    for k in ("dDw", "drho"):
        assert cancel[k] >= 1.0
        assert rel[k] <= 1e-5 * cancel[k], k
    assert np.allclose(b["dx0"], a["dx0"], rtol=2e-3, atol=1e-3 * np.abs(a["dx0"]).max())


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
    assert float(loss.detach()) == ref["loss"]
    assert float(Dw.grad) == pytest.approx(ref["dDw"] / L ** 2, rel=1e-14)
    assert float(rho.grad) == ref["drho"]
    assert np.allclose(x0.grad.numpy(), ref["dx0"], rtol=1e-14)
    pool.close()


def _gauss(n, x0, sigma, pw, pg):
    """The device's Gaussian initial condition (gaussian_ic_kernel): |x - x0|^2
    summed over x, y, z, then exp(-r2 / (2 sigma^2)) where there is tissue."""
    x = np.arange(n, dtype=np.float64) / n
    zz, yy, xx = np.meshgrid(x, x, x, indexing="ij")
    r2 = (xx - x0[0]) * (xx - x0[0]) + (yy - x0[1]) * (yy - x0[1]) + (zz - x0[2]) * (zz - x0[2])
    return np.where(pw + pg > 0, np.exp(-r2 / (2.0 * sigma * sigma)), 0.0), (xx, yy, zz)


def test_adjoint_equals_the_oracle_adjoint():
    """The FP64 device adjoint against the oracle's discrete adjoint
    (orc_loss_grad_f64 at the horizon, then orc_adjoint_step_dense_f64 back to
    t = 0, every state stored) on the same inputs: dL/dc0 as a whole field,
    dL/dDw, dL/drho, and dL/dx0 through the Gaussian initial condition.  Both
    hold the switches fixed and treat rounding as exact; they differ only in
    the order of the gradient sums (compensated on the device), so the
    tolerance is rounding-level: 1e-13 relative L2 for the field, 1e-12
    relative for the scalars."""
    pool, pw, pg, sched, t1, fl, R = _setup("f64", seed=7)
    sigma = 2.0 / N
    x0 = (0.52, 0.47, 0.5)
    c0, xs = _gauss(N, x0, sigma, pw, pg)
    Dw, Dg = _coeffs(R, 0.17)
    rho = 0.08
    pool.upload_dense("phi", c0)
    dev = pool.forward_adjoint(Dw, Dg, rho, sched.dt, NSTEPS, sigma=0.0, nsnapshots=6, grad_c0=True, **UC)
    u = O.rd_steps_dense(pw, pg, c0, Dw, Dg, rho, 1.0 / N, sched.dt, NSTEPS)
    lam_t = O.loss_grad(u, t1, fl, UC["t1_uc"], UC["t2_uc"], UC["slope"])
    lam0, drho, ddw = O.adjoint_dense(pw, pg, c0, Dw, Dg, rho, 1.0 / N, sched.dt, NSTEPS, lam_t)
    lik = O.log_likelihood(u, t1, fl, None, **UC)
    assert dev["loss"] == pytest.approx(-(lik[1] + lik[2]), rel=1e-12)
    g = dev["grad_c0"]
    assert np.count_nonzero(lam0) > 1000
    assert np.linalg.norm(g - lam0) <= 1e-13 * np.linalg.norm(lam0)
    assert dev["drho"] == pytest.approx(drho, rel=1e-12)
    assert dev["dDw"] == pytest.approx(ddw, rel=1e-12)
    # the magnitudes of the gradient terms (GBFK_ADJ_TERM_MAGNITUDES): the same
    # gradients bit for bit, and the oracle's sums of |term|
    pool.upload_dense("phi", c0)
    dev_m = pool.forward_adjoint(Dw, Dg, rho, sched.dt, NSTEPS, sigma=0.0, nsnapshots=6, term_magnitudes=True, **UC)
    assert all(dev_m[k] == dev[k] for k in ("loss", "dDw", "drho"))
    _, _, _, arho, adw = O.adjoint_dense(pw, pg, c0, Dw, Dg, rho, 1.0 / N, sched.dt, NSTEPS, lam_t, magnitudes=True)
    assert arho >= abs(drho) and adw >= abs(ddw)
    assert dev_m["drho_abs"] == pytest.approx(arho, rel=1e-12)
    assert dev_m["dDw_abs"] == pytest.approx(adw, rel=1e-12)
    # the origin: c0 = exp(-|x - x0|^2 / (2 sigma^2)), dc0/dx0_d = c0 (x_d - x0_d) / sigma^2
    dev_x = pool.forward_adjoint(Dw, Dg, rho, sched.dt, NSTEPS, x0=x0, sigma=sigma, nsnapshots=6, **UC)
    want = [np.sum(lam0 * c0 * (xs[d] - x0[d])) / sigma ** 2 for d in range(3)]
    assert np.allclose(dev_x["dx0"], want, rtol=1e-10, atol=1e-12 * np.abs(want).max())
    assert dev_x["drho"] == pytest.approx(drho, rel=1e-10)
    pool.close()


def test_adjoint_with_empty_blocks_skipped_equals_the_oracle():
    """At 64^3 most blocks outside the brain hold neither tissue nor tumour.
    The adjoint steps run only the blocks that can hold a domain cell and
    their face neighbours (the rest keep lambda = 0), and, when every empty
    block of the initial condition holds +0, the forward steps of the sweep
    run only the heavy blocks (the empty ones keep their +0).  Against the
    oracle's dense adjoint on one pool, in turn: tumour planted in a block
    outside the anatomy (a kEmpty cell with phi > 0 is inside the domain; no
    forward step skips), then the same anatomy without it (the forward steps
    skip, into buffers the first call wrote), then the first case again:
    dL/dc0 as a whole field, dL/dDw, dL/drho."""
    from gliomasolver_b200 import BlockPool

    n, bpd, nsteps = 64, 8, 30
    pw, pg, _ = make_anatomy(n, 4)
    clean = tumor_ic(n, (0.5, 0.5, 0.5), pw, pg)
    out = (pw + pg) == 0
    assert out[2:6, 2:6, 2:6].all() and out[:8, :8, :8].all()
    planted = clean.copy()
    planted[2:6, 2:6, 2:6] = 0.3     # tumour outside the anatomy, in corner block 0
    sched = make_schedule(0.2, 0.1, 100.0, L, bpd, "f64")
    rng = np.random.default_rng(3)
    u = O.rd_steps_dense(pw, pg, planted, sched.Dw, sched.Dg, sched.rho, 1.0 / n, sched.dt, nsteps)
    t1, fl = (u > 0.7).astype(float), (u > 0.25).astype(float)
    for m in (t1, fl):
        flip = rng.random(m.shape) < 0.02
        m[flip] = 1 - m[flip]
    with BlockPool(bpd ** 3, "f64") as pool:
        pool.set_uniform(bpd)
        pool.upload_dense("p_w", pw)
        pool.upload_dense("p_g", pg)
        pool.set_observations(t1, fl)
        for c0 in (planted, clean, planted):
            pool.upload_dense("phi", c0)
            dev = pool.forward_adjoint(sched.Dw, sched.Dg, sched.rho, sched.dt, nsteps, sigma=0.0, nsnapshots=5,
                                       grad_c0=True, **UC)
            u = O.rd_steps_dense(pw, pg, c0, sched.Dw, sched.Dg, sched.rho, 1.0 / n, sched.dt, nsteps)
            lam_t = O.loss_grad(u, t1, fl, UC["t1_uc"], UC["t2_uc"], UC["slope"])
            lam0, drho, ddw = O.adjoint_dense(pw, pg, c0, sched.Dw, sched.Dg, sched.rho, 1.0 / n, sched.dt, nsteps,
                                              lam_t)
            g = dev["grad_c0"]
            if c0 is planted:
                assert np.count_nonzero(lam0[:8, :8, :8]) > 0  # the planted tumour's block carries an adjoint
            assert np.count_nonzero(lam0 == 0) > n ** 3 // 4    # and most of the outside none
            assert np.linalg.norm(g - lam0) <= 1e-13 * np.linalg.norm(lam0)
            assert np.array_equal(g == 0, lam0 == 0)
            assert dev["drho"] == pytest.approx(drho, rel=1e-12)
            assert dev["dDw"] == pytest.approx(ddw, rel=1e-12)


@pytest.mark.skipif(not O.ref_available("f64"), reason="oracle/_ref is built only where the reference sources are")
def test_gradients_against_reference_forward_differences():
    """dL/dDw and dL/drho against central differences (relative step 1e-4) of
    the reference's own forward run (oracle/_ref/ref_harness_f64: the
    reference's ReactionDiffusionOperator and UpdateTumor through its
    BlockProcessing) followed by the likelihood."""
    pool, pw, pg, sched, t1, fl, R = _setup("f64", seed=8)
    c0 = tumor_ic(N, (0.5, 0.48, 0.51), pw, pg)
    Dw, Dg = _coeffs(R, 0.16)
    rho = 0.07
    pool.upload_dense("phi", c0)
    dev = pool.forward_adjoint(Dw, Dg, rho, sched.dt, NSTEPS, sigma=0.0, nsnapshots=4, **UC)

    def ref_loss(dw, rh):
        u = O.ref_uniform(pw, pg, c0, dw, 0.1 * dw, rh, sched.dt, NSTEPS, "f64")
        lik = O.log_likelihood(u, t1, fl, None, **UC)
        return -(lik[1] + lik[2])

    assert dev["loss"] == pytest.approx(ref_loss(Dw, rho), rel=1e-12)
    e = 1e-4 * Dw
    fd = (ref_loss(Dw + e, rho) - ref_loss(Dw - e, rho)) / (2 * e)
    assert dev["dDw"] == pytest.approx(fd, rel=1e-5)
    e = 1e-4 * rho
    fd = (ref_loss(Dw, rho + e) - ref_loss(Dw, rho - e)) / (2 * e)
    assert dev["drho"] == pytest.approx(fd, rel=1e-5)
    pool.close()


def test_config4_size_gradients_against_central_differences():
    """The config-4 problem at its full size: 128^3, Dw = 0.2 cm^2/day and
    rho = 0.012/day for T = 300 days (9091 steps), 64 checkpoint buffers,
    observations from a seeded ground-truth run thresholded at 0.7 / 0.25 with
    2% label noise, gradients at Dw = 0.18, rho = 0.014 and an origin 2 cells
    off.  FP64 state: dDw and drho against central differences with relative
    step 1e-4 of the forward map (FP64 device steps, equal bit for bit to the
    reference's operator sweep), dx0 against relative step 1e-7 (a larger
    shift moves voxels across a likelihood threshold); no voxel may cross a
    threshold between the two runs of a quotient.  FP32 state with FP64 sums:
    against the FP64 gradients."""
    from gliomasolver_b200 import BlockPool
    from gliomasolver_b200.anatomy import make_anatomy, pick_origin
    from gliomasolver_b200.gradcheck import check_gradients, synthetic_observations

    n, bpd = 128, 16
    p_w, p_g, _ = make_anatomy(n, 0)
    x_gt = pick_origin(p_w, 0)[0]
    x0 = [float(min(1.0, v + 2.0 / n)) for v in x_gt]
    res = {}
    for prec in ("f64", "f32"):
        R = np.float64 if prec == "f64" else np.float32
        s = make_schedule(0.2, 0.012, 300.0, L, bpd, prec)
        assert s.nsteps > 9000
        with BlockPool(bpd ** 3, prec) as pool:
            pool.set_uniform(bpd)
            pool.upload_dense("p_w", p_w.astype(R))
            pool.upload_dense("p_g", p_g.astype(R))
            synthetic_observations(pool, tumor_ic(n, x_gt, p_w, p_g), s.Dw, s.rho, s.dt, s.nsteps, seed=17)
            Dw = float(R(R(0.18) / R(L * L)))
            if prec == "f64":
                res[prec] = chk = check_gradients(pool, p_w, p_g, Dw, 0.014, s.dt, s.nsteps, x0, 2.0 / n,
                                                  nsnapshots=64, **UC)
                print(chk)
                assert chk["forward_steps"] < 2.8 * s.nsteps
                for k in ("dDw", "drho"):
                    assert chk["crossings"][k] == 0, chk
                    assert chk["rel_err"][k] <= 1e-5, (k, chk)
                # x0: a shift above 1e-7 moves voxels across a threshold, and at
                # 1e-7 the quotient resolves the loss's last place only to a few
                # 1e-4 relative; the tolerance is five times that resolution
                # (at least 1e-4), and the chain rule through dL/dc0 is tight
                for d in range(3):
                    k = f"dx0[{d}]"
                    assert chk["crossings"][k] == 0, chk
                    assert chk["rel_err"][k] <= max(1e-4, 5 * chk["fd_resolution"][k]), (k, chk)
                assert chk["chain_rule_rel_err"] <= 1e-10, chk
            else:
                res[prec] = pool.forward_adjoint(Dw, float(R(0.1 * np.float64(Dw))), 0.014, s.dt, s.nsteps, x0=x0,
                                                 sigma=2.0 / n, nsnapshots=64, **UC)
    a, b = res["f64"]["adjoint"], res["f32"]
    rel = {k: abs(b[k] - a[k]) / abs(a[k]) for k in ("dDw", "drho")}
    rel["loss"] = abs(b["loss"] - res["f64"]["loss"]) / abs(res["f64"]["loss"])
    print({"fp32_vs_fp64_rel": rel})
    assert rel["loss"] <= 1e-4


def test_autograd_initial_field():
    """tumor_loss with an explicit initial field: c0.grad is the adjoint state
    at t = 0 (gbfk_forward_adjoint's grad_c0), Dw and rho get their gradients."""
    import torch

    from gliomasolver_b200.autograd import tumor_loss

    pool, pw, pg, sched, t1, fl, R = _setup("f64", seed=9)
    c0n = tumor_ic(N, (0.5, 0.47, 0.52), pw, pg)
    c0 = torch.tensor(c0n, dtype=torch.float64, requires_grad=True)
    Dw = torch.tensor(0.15, dtype=torch.float64, requires_grad=True)
    rho = torch.tensor(0.08, dtype=torch.float64, requires_grad=True)
    loss = tumor_loss(pool, Dw, rho, None, L, sched.dt, NSTEPS, 0.0, nsnapshots=7, c0=c0)
    (2.0 * loss).backward()
    Dwr, Dgr = _coeffs(R, 0.15)
    pool.upload_dense("phi", c0n)
    ref = pool.forward_adjoint(Dwr, Dgr, 0.08, sched.dt, NSTEPS, sigma=0.0, nsnapshots=7, grad_c0=True, **UC)
    assert float(loss.detach()) == ref["loss"]
    assert np.array_equal(c0.grad.numpy(), 2.0 * ref["grad_c0"])
    assert float(rho.grad) == 2.0 * ref["drho"]
    assert float(Dw.grad) == pytest.approx(2.0 * ref["dDw"] / L ** 2, rel=1e-14)
    pool.close()


def test_adjoint_with_a_roi_matches_central_differences():
    """With a ROI the loss sums over its points only, each as often as it is
    listed (HGG_Likelihood.cpp:97-124): the FP64 gradients against central
    differences (relative step 1e-4) of the same ROI loss, and dL/dc0 against
    the oracle's adjoint of the count-weighted loss gradient."""
    pool, pw, pg, sched, t1, fl, R = _setup("f64", seed=11)
    rng = np.random.default_rng(12)
    pts = rng.integers(0, N, (N ** 3 // 3, 3)).astype(np.int32)
    roi = np.concatenate([pts, pts[: N ** 3 // 20]])          # some points listed twice
    pool.set_observations(t1, fl, roi=roi)
    c0 = tumor_ic(N, (0.51, 0.49, 0.5), pw, pg)
    Dw, Dg = _coeffs(R, 0.16)
    rho = 0.07
    pool.upload_dense("phi", c0)
    dev = pool.forward_adjoint(Dw, Dg, rho, sched.dt, NSTEPS, sigma=0.0, nsnapshots=5, grad_c0=True, **UC)

    def loss(dw, rh):
        pool.upload_dense("phi", c0)
        pool.rd_step(dw, float(R(0.1 * np.float64(dw))), rh, sched.dt, NSTEPS)
        lik = pool.log_likelihood(**UC)
        return -(lik[1] + lik[2])

    assert dev["loss"] == pytest.approx(loss(Dw, rho), rel=1e-13)
    e = 1e-4 * Dw
    assert dev["dDw"] == pytest.approx((loss(Dw + e, rho) - loss(Dw - e, rho)) / (2 * e), rel=1e-5)
    e = 1e-4 * rho
    assert dev["drho"] == pytest.approx((loss(Dw, rho + e) - loss(Dw, rho - e)) / (2 * e), rel=1e-5)
    count = np.zeros((N, N, N))
    np.add.at(count, (roi[:, 2], roi[:, 1], roi[:, 0]), 1.0)
    u = O.rd_steps_dense(pw, pg, c0, Dw, Dg, rho, 1.0 / N, sched.dt, NSTEPS)
    lam_t = count * O.loss_grad(u, t1, fl, UC["t1_uc"], UC["t2_uc"], UC["slope"])
    lam0, drho, ddw = O.adjoint_dense(pw, pg, c0, Dw, Dg, rho, 1.0 / N, sched.dt, NSTEPS, lam_t)
    assert np.linalg.norm(dev["grad_c0"] - lam0) <= 1e-13 * np.linalg.norm(lam0)
    assert dev["dDw"] == pytest.approx(ddw, rel=1e-12)
    pool.close()
