"""The oracle's restatement of the discrete adjoint (orc_adjoint_step_dense_f64)
and of the loss gradient (orc_loss_grad_f64), checked on the CPU against
central differences of the oracle's own forward steps and likelihood: the
reference for the device adjoint beside finite differences."""
import numpy as np

from gliomasolver_b200.anatomy import make_case
from gliomasolver_b200.schedule import make_schedule
from oracle import oracle as O


def _case():
    n = 16
    pw, pg, _, _ = make_case(n, 2)
    s = make_schedule(0.3, 0.1, 150.0, 25.6, n // 8, "f64")
    x = np.arange(n) / n
    zz, yy, xx = np.meshgrid(x, x, x, indexing="ij")
    r2 = (xx - 0.5) ** 2 + (yy - 0.5) ** 2 + (zz - 0.5) ** 2
    c0 = np.where(pw + pg > 0, 0.45 * np.exp(-r2 / 0.02), 0.0)
    return pw, pg, c0, s


def test_adjoint_matches_central_differences():
    pw, pg, c0, s = _case()
    nsteps = 12
    w = np.random.default_rng(0).standard_normal(c0.shape)

    def loss(phi0, Dw=s.Dw, rho=s.rho):
        u = O.rd_steps_dense(pw, pg, phi0, Dw, 0.1 * Dw, rho, s.h, s.dt, nsteps)
        return float(np.sum(w * u))

    lam0, drho, ddw = O.adjoint_dense(pw, pg, c0, s.Dw, 0.1 * s.Dw, s.rho, s.h, s.dt, nsteps, w)
    cells = np.argwhere((c0 > 0.05) & (c0 < 0.4))[::7][:8]
    assert len(cells) == 8
    for c in map(tuple, cells):
        e = np.zeros_like(c0)
        e[c] = 1e-6
        fd = (loss(c0 + e) - loss(c0 - e)) / 2e-6
        assert abs(fd - lam0[c]) <= 1e-6 * abs(fd) + 1e-9, c
    er, ed = 1e-6 * s.rho, 1e-6 * s.Dw
    fd_rho = (loss(c0, rho=s.rho + er) - loss(c0, rho=s.rho - er)) / (2 * er)
    fd_dw = (loss(c0, Dw=s.Dw + ed) - loss(c0, Dw=s.Dw - ed)) / (2 * ed)
    assert abs(drho - fd_rho) <= 1e-6 * abs(fd_rho)
    assert abs(ddw - fd_dw) <= 1e-6 * abs(fd_dw)


def test_loss_gradient_matches_central_differences():
    rng = np.random.default_rng(4)
    n = 8
    u = rng.uniform(0, 1, (n, n, n))
    t1c = (rng.uniform(0, 1, u.shape) > 0.6).astype(float)
    flair = (rng.uniform(0, 1, u.shape) > 0.4).astype(float)
    g = O.loss_grad(u, t1c, flair, 0.7, 0.25, 2.0)
    for c in map(tuple, rng.integers(0, n, (12, 3))):
        if min(abs(u[c] - 0.7), abs(u[c] - 0.25)) < 1e-3:
            continue  # the likelihood is discontinuous at the thresholds
        e = np.zeros_like(u)
        e[c] = 1e-6
        lp = O.log_likelihood(u + e, t1c, flair)
        lm = O.log_likelihood(u - e, t1c, flair)
        fd = -((lp[1] + lp[2]) - (lm[1] + lm[2])) / 2e-6
        assert abs(fd - g[c]) <= 1e-5 * max(abs(fd), 1e-3), (c, fd, g[c])


def test_origin_gradient_through_the_initial_condition():
    """dL/dx0 = sum_i lambda0_i dc0_i/dx0 with c0 = exp(-|x - x0|^2 / (2 sigma^2))
    where there is tissue (the Gaussian initial condition of the workloads),
    against central differences of x0."""
    from gliomasolver_b200.anatomy import tumor_ic

    pw, pg, _, s = _case()
    n, nsteps = pw.shape[0], 10
    w = np.random.default_rng(1).standard_normal(pw.shape)
    x0 = np.array([0.47, 0.52, 0.49])
    sigma = 2.0 / n
    x = np.arange(n) / n
    zz, yy, xx = np.meshgrid(x, x, x, indexing="ij")

    def loss(p):
        c0 = tumor_ic(n, p, pw, pg)
        return float(np.sum(w * O.rd_steps_dense(pw, pg, c0, s.Dw, s.Dg, s.rho, s.h, s.dt, nsteps)))

    c0 = tumor_ic(n, x0, pw, pg)
    lam0, _, _ = O.adjoint_dense(pw, pg, c0, s.Dw, s.Dg, s.rho, s.h, s.dt, nsteps, w)
    grad = [float(np.sum(lam0 * c0 * (g - x0[d]) / sigma ** 2)) for d, g in enumerate((xx, yy, zz))]
    for d in range(3):
        e = np.zeros(3)
        e[d] = 1e-7
        fd = (loss(x0 + e) - loss(x0 - e)) / 2e-7
        assert abs(fd - grad[d]) <= 1e-5 * abs(fd) + 1e-6, (d, fd, grad[d])


def test_transposed_step_amplifies_next_to_the_no_flux_switch():
    """Why config 5's gradients are ill-conditioned: the no-flux switch
    (ReactionDiffusionOperator.h:166-181) doubles the coefficient opposite a
    neighbour whose chf is below 0.1, so the step's transpose is not a
    contraction.  With the state positive in every tissue cell (mu = lambda
    there), one adjoint step of lambda = 1 gives the column sums of the step's
    Jacobian: they exceed 1 + dt rho (the bound of its row sums) next to
    those faces, and repeated steps grow lambda."""
    n = 32
    pw, pg, _, _ = make_case(n, 3)
    s = make_schedule(0.23, 0.0057, 250.0, 25.6, n // 8, "f64")
    tissue = (pw + pg) > 0
    phi = np.where(tissue, 1e-300, 0.0)
    lam = np.ones_like(phi)
    col = O.adjoint_dense(pw, pg, phi, s.Dw, s.Dg, s.rho, s.h, s.dt, 1, lam)[0]
    bound = 1.0 + s.dt * s.rho
    assert col[tissue].max() > 1.04 * bound
    assert np.count_nonzero(col[tissue] > bound * (1 + 1e-12)) > 1000
    lam = O.adjoint_dense(pw, pg, phi, s.Dw, s.Dg, s.rho, s.h, s.dt, 200, np.ones_like(phi))[0]
    assert lam.max() > 2.0
