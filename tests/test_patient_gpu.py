"""A patient case through the device path: Matrix files mapped by
gbfk_map_anatomy (the reference's _ic), uploaded to a block pool and stepped
on the GPU with the schedule of the mapped characteristic length; the
result must equal the oracle's steps on the same cells bit for bit."""
import numpy as np
import pytest

from gliomasolver_b200 import BlockPool, patient
from gliomasolver_b200.schedule import make_schedule
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _volumes(shape, seed):
    """A smooth brain-like volume: tissue inside an ellipsoid, CSF in a core."""
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(*(np.linspace(-1, 1, s) for s in shape), indexing="ij")
    r = np.sqrt((x / 0.9) ** 2 + (y / 0.8) ** 2 + (z / 0.85) ** 2)
    wm = np.clip(1.2 - r, 0, 1) * rng.uniform(0.8, 1.0, shape)
    gm = np.clip(1.0 - np.abs(r - 0.8) * 3, 0, 1) * rng.uniform(0.8, 1.0, shape)
    csf = np.where(r < 0.15, 1.0, 0.0) + np.where(r > 1.0, 0.3, 0.0)
    return gm, wm, csf


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_patient_case_steps_like_the_oracle(gbfk_lib, tmp_path, prec):
    bpd, tic = 4, (0.3 + 0.004, 0.5 - 0.006, 0.4 + 0.002)
    for k, v in zip(("GM", "WM", "CSF"), _volumes((36, 44, 40), 1)):
        patient.write_matrix(tmp_path / f"P_{k}.dat", v, type_id=1)
    a = patient.load_patient(tmp_path / "P_", bpd, tic, prec)
    assert np.count_nonzero(a.phi) > 0 and a.L_cm == pytest.approx(4.4)
    s = make_schedule(0.13, 0.025, 150.0, a.L_cm, bpd, prec)
    n = 8 * bpd
    steps = min(int(s.nsteps), 60)
    with BlockPool(bpd ** 3, prec) as pool:
        pool.set_uniform(bpd)
        pool.upload_dense("p_w", a.p_w)
        pool.upload_dense("p_g", a.p_g)
        pool.upload_dense("phi", a.phi)
        pool.rd_step(s.Dw, s.Dg, s.rho, s.dt, steps, check_nan=True)
        out = pool.download_dense("phi")
    want = O.rd_steps_dense(a.p_w, a.p_g, a.phi, s.Dw, s.Dg, s.rho, s.h, s.dt, steps)
    assert out.shape == (n, n, n)
    assert np.array_equal(out, want)


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_batch_ball_tumour_equals_the_mapping(gbfk_lib, prec):
    """GBFK_IC_BALL samples of a batch start from the reference's smoothed
    ball: with no steps their state is gbfk_map_anatomy's phi bit for bit
    (tumours inside, at the edge of and outside the tissue, and one next
    to the domain's corner), and after their steps it equals a block pool
    stepped from that phi."""
    from gliomasolver_b200.tmcmc import Batch, StageSample, to_gbfk_samples

    bpd = 4
    gm, wm, csf = _volumes((36, 44, 40), 2)
    tics = [(0.304, 0.494, 0.402), (0.5 + 0.003, 0.5 - 0.007, 0.5 + 0.001), (0.12, 0.2, 0.31),
            (0.002, 0.004, 0.001), (0.72, 0.61, 0.55)]
    maps = [patient.map_anatomy(gm, wm, csf, bpd, t, prec) for t in tics]
    a0 = maps[0]
    assert all(np.array_equal(m.p_w, a0.p_w) for m in maps)
    assert sum(np.count_nonzero(m.phi) for m in maps) > 0
    stage = [StageSample(0.13, 0.025, 40.0, t) for t in tics] * 2
    samples, scheds = to_gbfk_samples(stage, bpd, prec, a0.L_cm, ic="ball")
    for i in range(len(tics)):
        samples[i].nsteps = 0
    steps = [int(samples[i].nsteps) for i in range(len(stage))]
    with Batch(bpd, len(stage), prec) as batch:
        batch.set_anatomy(0, a0.p_w, a0.p_g)
        batch.set_samples(samples)
        batch.run(0)
        got = [batch.download(i) for i in range(len(stage))]
    for i, m in enumerate(maps):
        assert np.array_equal(got[i], m.phi), i
    s = scheds[len(tics)]
    for i, m in enumerate(maps):
        j = len(tics) + i
        with BlockPool(bpd ** 3, prec) as pool:
            pool.set_uniform(bpd)
            pool.upload_dense("p_w", a0.p_w)
            pool.upload_dense("p_g", a0.p_g)
            pool.upload_dense("phi", m.phi)
            pool.rd_step(s.Dw, s.Dg, s.rho, s.dt, steps[j], check_nan=True)
            assert np.array_equal(got[j], pool.download_dense("phi")), j
