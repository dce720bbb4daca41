"""The in-process TMCMC driver (gliomasolver_b200.tmcmc.tmcmc) on problems
with known answers, on CPU: the tempering schedule, the weights' evidence
estimate and the posterior moments; and the glioma model on the GPU."""
import numpy as np
import pytest

from gliomasolver_b200.tmcmc import TMCMCOptions, next_exponent, tmcmc


def test_next_exponent_hits_the_target_cov():
    """The reference's grid search stops at the first exponent whose
    (COV - 1)^2 is within opt.Tol: |COV - 1| <= 1e-3 at the engine's default
    1e-6, and far closer at the 1e-12 of tmcmc_glioma.par."""
    rng = np.random.default_rng(1)
    F = rng.normal(0, 50, 1000)
    for tol, rel in ((1e-6, 1e-3), (1e-12, 1e-6)):
        p1 = next_exponent(F, 0.0, 1.0, tol)
        w = np.exp((F - F.max()) * p1)
        q = w / w.sum()
        assert 0 < p1 < 1
        assert q.std(ddof=1) / q.mean() == pytest.approx(1.0, rel=rel)
    # a flat likelihood never reaches the target COV: the reference then
    # steps the exponent by 1e-5 (calculate_statistics, tmcmc_stats.c:611-617)
    assert next_exponent(np.zeros(10), 0.3, 1.0) == pytest.approx(0.3 + 1e-5, abs=1e-15)
    # a root above 1 ends the tempering
    assert next_exponent(rng.normal(0, 0.5, 1000), 0.3, 1.0) == 1.0


def test_gaussian_posterior_and_evidence():
    """Uniform prior on a box, normalised Gaussian likelihood well inside it:
    the evidence is 1 / box volume and the posterior is the Gaussian."""
    mu = np.array([0.3, -0.2])
    cov = np.array([[0.02, 0.006], [0.006, 0.01]])
    icov = np.linalg.inv(cov)
    lognorm = -0.5 * np.log(np.linalg.det(2 * np.pi * cov))
    lower, upper = np.array([-2.0, -2.0]), np.array([2.0, 2.0])

    def loglik(th):
        d = th - mu
        return lognorm - 0.5 * np.einsum("ni,ij,nj->n", d, icov, d)

    res = tmcmc(loglik, lower, upper, TMCMCOptions(pop_size=4000, seed=3))
    assert res.p[0] == 0 and res.p[-1] == 1 and all(np.diff(res.p) > 0)
    assert res.log_evidence == pytest.approx(-np.log(16.0), abs=0.1)
    assert np.allclose(res.theta.mean(axis=0), mu, atol=0.02)
    assert np.allclose(np.cov(res.theta.T), cov, atol=0.004)
    assert res.evaluations == 4000 * len(res.p)


def test_penalty_for_failed_evaluations():
    """NaN log-likelihoods count as the reference's 1e12 penalty: such
    regions end up with no samples."""
    def loglik(th):
        f = -0.5 * np.sum((th - 0.5) ** 2, axis=1) / 0.01
        f[th[:, 0] < 0] = np.nan
        return f

    res = tmcmc(loglik, [-1, -1], [1, 1], TMCMCOptions(pop_size=1000, seed=5))
    assert np.all(res.theta[:, 0] >= 0)


@pytest.mark.gpu
def test_glioma_model_calibration_runs_on_the_batch(gbfk_lib):
    """A short calibration at 32^3: observations from a ground-truth solve,
    the population's forward solves and likelihoods in batches; the
    ground truth scores higher than a far-off parameter set, and the
    posterior concentrates around the truth's Dw*T and rho*T."""
    from gliomasolver_b200.anatomy import make_anatomy
    from gliomasolver_b200.tmcmc import GliomaModel

    n = 32
    pw, pg, _ = make_anatomy(n, 1)
    truth = np.log([0.15, 0.06, 0.06 * 40.0 ** 2, 0.5, 0.5, 0.5, 0.019, 0.85, 0.7, 0.25, 2.0])
    model = GliomaModel(pw, pg, np.zeros((n,) * 3), np.zeros((n,) * 3), max_samples=256)
    try:
        # synthetic masks from the truth's own state
        from gliomasolver_b200.tmcmc import StageSample, to_gbfk_samples

        Dw, rho, tend, x0 = 0.15, 0.06, 40.0, (0.5, 0.5, 0.5)
        samples, _ = to_gbfk_samples([StageSample(Dw, rho, tend, x0)], n // 8, "f32")
        model.batch.set_samples(samples)
        model.batch.run(0)
        u = model.batch.download(0).astype(np.float64)
        model.batch.set_observations((u > 0.7).astype(float), (u > 0.25).astype(float))
        far = truth.copy()
        far[1] = np.log(0.01)
        F = model(np.stack([truth, far]))
        assert np.all(np.isfinite(F)) and F[0] > F[1]
        lower, upper = truth.copy(), truth.copy()
        lower[:2] -= 1.0
        upper[:2] += 1.0
        res = tmcmc(model, lower, upper, TMCMCOptions(pop_size=128, max_stages=7, seed=2))
        assert len(res.p) >= 2 and np.all(np.isfinite(res.loglik))
        best = res.theta[np.argmax(res.loglik)]
        assert abs(best[1] - truth[1]) < 0.5
    finally:
        model.close()
