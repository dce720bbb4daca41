"""Batched TMCMC-stage forward solves: every sample of a batch must equal the
same sample solved alone (gbfk_rd_step on a BlockPool) bit for bit, whatever
the kernel choice (the pipelined step over all active samples, or the
per-block kernel with 1, 2 or 4 samples per CTA), with uneven horizons and
several anatomies."""
import numpy as np
import pytest

from gliomasolver_b200.anatomy import make_anatomy
from gliomasolver_b200.schedule import make_schedule
from gliomasolver_b200.tmcmc import sample_stage, to_gbfk_samples


def test_stage_sampling_matches_the_configured_ranges():
    """Config 3: Dw log-U[0.02, 0.3], rho log-U[0.002, 0.2], T U[30, 300] at
    128^3 give horizons from about 10^2 to about 1.4*10^4 steps."""
    p_w, _, _ = make_anatomy(32, 0)
    stage = sample_stage(512, p_w, seed=3)
    Dw = np.array([s.Dw_cm2_day for s in stage])
    rho = np.array([s.rho_day for s in stage])
    T = np.array([s.tend_day for s in stage])
    assert Dw.min() >= 0.02 and Dw.max() <= 0.3
    assert rho.min() >= 0.002 and rho.max() <= 0.2
    assert T.min() >= 30 and T.max() <= 300
    steps = [make_schedule(s.Dw_cm2_day, s.rho_day, s.tend_day, 25.6, 16, "f32").nsteps for s in stage[:64]]
    assert 50 < min(steps) and max(steps) < 15000
    assert stage == sample_stage(512, p_w, seed=3)


@pytest.mark.gpu
@pytest.mark.parametrize("prec,bpd", [("f32", 4), ("f64", 4), ("f32", 8)])
def test_batch_equals_sequential_solves(gbfk_lib, prec, bpd):
    """Every sample of a batch (two anatomies, uneven horizons) equals its own
    solve bit for bit, for every kernel the batch can run; at 64^3 most
    blocks are empty, which the pipelined batch step skips after its first
    step."""
    from gliomasolver_b200 import BlockPool
    from gliomasolver_b200.tmcmc import Batch

    R = np.float64 if prec == "f64" else np.float32
    n = 8 * bpd
    anat = [make_anatomy(n, seed) for seed in (0, 5)]
    anat = [(a[0].astype(R), a[1].astype(R)) for a in anat]
    stage = sample_stage(10, anat[0][0], seed=11, tend_range=(2.0, 40.0))
    which = [i % 2 for i in range(10)]
    samples, scheds = to_gbfk_samples(stage, bpd, prec, anatomy=which)
    assert len({s.nsteps for s in scheds}) > 5

    # the initial conditions the batch builds (a run of 0 steps)
    zero, _ = to_gbfk_samples(stage, bpd, prec, anatomy=which)
    for r in zero:
        r.nsteps = 0
    with Batch(bpd, 10, prec, max_anatomies=2) as b:
        for i, (pw, pg) in enumerate(anat):
            b.set_anatomy(i, pw, pg)
        b.set_samples(zero)
        b.run(1)
        c0 = [b.download(i) for i in range(10)]
        results = {}
        for spc in (1, 2, 4, -1, 0):
            b.set_samples(samples)
            b.run(spc)
            results[spc] = [b.download(i) for i in range(10)]
            if spc == 0:
                # the autotuner ran every candidate (each launch shape of the
                # pipelined step, 1/2/4 samples per CTA) on real steps
                assert b.samples_per_cta in (-1, 1, 2, 4)
            assert (b.tile_shape == (0, 0, 0)) == (b.samples_per_cta != -1)
            if max(s.nsteps for s in scheds) > 60:
                assert b.graph_count >= 1   # the steps after the autotuner replay as CUDA graphs

    for i in range(10):
        pw, pg = anat[which[i]]
        s = scheds[i]
        with BlockPool(bpd ** 3, prec) as pool:
            pool.set_uniform(bpd)
            pool.upload_dense("p_w", pw)
            pool.upload_dense("p_g", pg)
            pool.upload_dense("phi", c0[i])
            pool.rd_step(s.Dw, s.Dg, s.rho, s.dt, s.nsteps)
            want = pool.download_dense("phi")
        assert c0[i].max() > 0.5
        for spc, res in results.items():
            assert np.array_equal(res[i], want), (i, spc)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_batch_likelihood_equals_per_sample_likelihood(gbfk_lib, prec):
    """The likelihood step run on the device after a batch equals, for every
    sample, the dump + likelihood of the same sample solved alone (same
    observations: T1c / FLAIR masks, PET signal, ROI subset)."""
    from gliomasolver_b200 import BlockPool
    from gliomasolver_b200.tmcmc import Batch

    R = np.float64 if prec == "f64" else np.float32
    bpd, n = 4, 32
    pw, pg, _ = make_anatomy(n, 2)
    pw, pg = pw.astype(R), pg.astype(R)
    stage = sample_stage(6, pw, seed=4, tend_range=(5.0, 30.0))
    samples, scheds = to_gbfk_samples(stage, bpd, prec)
    rng = np.random.default_rng(9)
    t1 = (rng.random((n, n, n)) < 0.05).astype(float)
    fl = np.maximum(t1, (rng.random((n, n, n)) < 0.1)).astype(float)
    pet = rng.random((n, n, n)) * 0.3
    roi = rng.integers(0, n, (200, 3))
    kw = dict(step_pet=2, step_mri=1)
    with Batch(bpd, 6, prec) as b:
        b.set_anatomy(0, pw, pg)
        zero, _ = to_gbfk_samples(stage, bpd, prec)
        for r in zero:
            r.nsteps = 0
        b.set_samples(zero)
        b.run(1)
        c0 = [b.download(i) for i in range(6)]
        b.set_samples(samples)
        b.run(0)
        b.set_observations(t1, fl, pet, roi)
        got = b.log_likelihood(**kw)
    with BlockPool(bpd ** 3, prec) as pool:
        pool.set_uniform(bpd)
        pool.upload_dense("p_w", pw)
        pool.upload_dense("p_g", pg)
        pool.set_observations(t1, fl, pet, roi)
        for i, s in enumerate(scheds):
            pool.upload_dense("phi", c0[i])
            pool.rd_step(s.Dw, s.Dg, s.rho, s.dt, s.nsteps)
            assert np.array_equal(got[i], pool.log_likelihood(**kw)), i
    assert np.all(np.isfinite(got)) and len({tuple(r) for r in got}) == 6
