"""The oracle (CPU restatement) pinned against the reference.

The golden fixtures were produced by the reference's own operators
(oracle/_ref, see tests/golden/make_golden.py); the restatement must
reproduce them bit for bit.  Where oracle/_ref is present the restatement is
also compared with it directly on fresh inputs.
"""
import hashlib

import numpy as np
import pytest

from gliomasolver_b200.anatomy import make_case
from gliomasolver_b200.schedule import make_schedule
from oracle import oracle as O


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


def _inputs(fx):
    n, seed, prec = int(fx["n"]), int(fx["seed"]), str(fx["precision"])
    R = np.float64 if prec == "f64" else np.float32
    pw, pg, c0, _ = make_case(n, seed)
    pw, pg, c0 = (a.astype(R) for a in (pw, pg, c0))
    h = hashlib.sha256()
    for a in (pw, pg, c0):
        h.update(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    assert h.hexdigest() == str(fx["input_sha"]), "synthetic inputs drifted from the fixture"
    return pw, pg, c0, R


@pytest.mark.parametrize("name", ["rhs_n32_f64", "rhs_n32_f32"])
def test_rhs_matches_reference(golden, name):
    fx = golden(name)
    pw, pg, c0, R = _inputs(fx)
    out = O.rd_rhs_dense(pw, pg, c0, fx["Dw"], fx["Dg"], fx["rho"], fx["h"])
    assert np.array_equal(out.astype(np.float64), fx["out"])


@pytest.mark.parametrize("name", ["steps_n32_f64", "steps_n32_f32", "steps_n16_f64_fast"])
def test_steps_match_reference(golden, name):
    fx = golden(name)
    pw, pg, c0, R = _inputs(fx)
    out = O.rd_steps_dense(pw, pg, c0, fx["Dw"], fx["Dg"], fx["rho"], fx["h"], fx["dt"], int(fx["nsteps"]))
    assert np.array_equal(out.astype(np.float64), fx["out"])


def test_config1_full_run_matches_reference(golden):
    """64^3, FP64, T = 150 d at the reference's CFL dt (739 steps)."""
    fx = golden("config1_n64_f64")
    assert int(fx["nsteps"]) == 739
    pw, pg, c0, R = _inputs(fx)
    out = O.rd_steps_dense(pw, pg, c0, fx["Dw"], fx["Dg"], fx["rho"], fx["h"], fx["dt"], int(fx["nsteps"]))
    assert _sha(out) == str(fx["output_sha"])
    assert np.array_equal(out[::4, ::4, ::4], fx["out_sub"])


def test_schedule_matches_driver():
    """dt and the step count of Glioma_ReactionDiffusion::run (:300-321)."""
    s = make_schedule(0.13, 0.025, 150.0, 25.6, 8, "f64")
    assert s.nsteps == 739
    assert s.Dg == pytest.approx(0.1 * s.Dw)
    assert s.dt == 0.99 * (1 / 64) * (1 / 64) / (6 * s.Dw)
    s32 = make_schedule(0.13, 0.025, 150.0, 25.6, 8, "f32")
    assert np.float32(s32.dt) == s32.dt
    # config 2's 256^3 schedule: Dw = 0.2, T = 300 d
    s2 = make_schedule(0.2, 0.05, 300.0, 25.6, 32, "f32")
    assert 35000 < s2.nsteps < 37500


@pytest.mark.skipif(not O.ref_available("f64"), reason="oracle/_ref (reference build) not present")
@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("n,seed,steps", [(8, 11, 7), (16, 5, 13)])
def test_restatement_vs_reference_fresh_inputs(prec, n, seed, steps):
    # MRAG grids need a power-of-two number of blocks per direction
    R = np.float64 if prec == "f64" else np.float32
    pw, pg, c0, _ = make_case(n, seed)
    # stress the branches: a CSF hole next to tumour, and an initial value > 1
    pw[n // 2, n // 2, : n // 4] = 0.0
    pg[n // 2, n // 2, : n // 4] = 0.0
    c0[n // 2, n // 2, n // 4] = 1.5
    pw, pg, c0 = (a.astype(R) for a in (pw, pg, c0))
    s = make_schedule(0.2, 0.1, 100.0, 25.6, n // 8, prec)
    ref = O.ref_uniform(pw.astype(np.float64), pg.astype(np.float64), c0.astype(np.float64), s.Dw, s.Dg,
                        s.rho, s.dt, steps, prec)
    mine = O.rd_steps_dense(pw, pg, c0, s.Dw, s.Dg, s.rho, s.h, s.dt, steps)
    assert np.array_equal(mine.astype(np.float64), ref)
