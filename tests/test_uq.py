"""The UQ end of the path: the finest-uniform dump of phi and the
log-likelihood of the observations, against the oracle and (for the
likelihood) the reference's own likelihood program."""
import numpy as np
import pytest

from gliomasolver_b200.anatomy import make_case
from oracle import oracle as O
from topology_util import LAB_GHOSTS

PARAMS = dict(pet_sigma2=0.000361, pet_scale=0.85, t1_uc=0.7, t2_uc=0.25, slope=2.0)


def _observations(n, seed):
    rng = np.random.default_rng(seed)
    pw, pg, c0, _ = make_case(n, seed)
    model = np.clip(c0 + 0.3 * rng.random((n, n, n)) * (pw + pg > 0), 0, 1)
    t1 = (rng.random((n, n, n)) < 0.3).astype(float)
    fl = (rng.random((n, n, n)) < 0.5).astype(float)
    pet = np.where(rng.random((n, n, n)) < 0.4, rng.random((n, n, n)), 0.0)
    roi = np.stack(np.nonzero(pw + pg > 0)[::-1], 1)[::7]
    return pw, pg, model, t1, fl, pet, roi


@pytest.mark.skipif(not O.REF_DIR.joinpath("likelihood").exists(), reason="reference likelihood not built")
@pytest.mark.parametrize("use_roi", [False, True])
def test_oracle_likelihood_matches_reference_program(use_roi):
    """HGG_Likelihood built from the reference sources prints the terms with
    6 decimals; the restatement (long double) must agree to that precision."""
    n = 24
    _, _, model, t1, fl, pet, roi = _observations(n, 3)
    r = roi if use_roi else None
    mine = O.log_likelihood(model, t1, fl, pet, roi=r, step_pet=3, step_mri=2, **PARAMS)
    ref, out = O.ref_likelihood(model, t1, fl, pet, roi=r, step_pet=3, step_mri=2, **PARAMS)
    line = [ln for ln in out.splitlines() if ln.startswith("L_Pet=")][0]
    vals = [float(x.split("=")[1]) for x in line.replace(" ", "").split(",")]
    assert np.allclose(mine, vals, rtol=0, atol=1e-6)
    assert abs(-mine.sum() - ref) < 1e-5


def _mixed_level_blocks():
    """A level-3 grid (8^3 blocks) with one block split into eight level-4
    blocks and one family of eight level-3 blocks merged into a level-2 block;
    trivial ghost lists (the dump reads none)."""
    blocks = []
    for bz in range(8):
        for by in range(8):
            for bx in range(8):
                if (bx, by, bz) == (5, 5, 5):
                    for c in range(8):
                        cx, cy, cz = c & 1, (c >> 1) & 1, c >> 2
                        blocks.append((4, (2 * bx + cx, 2 * by + cy, 2 * bz + cz)))
                elif bx < 2 and by < 2 and bz < 2:
                    if (bx, by, bz) == (0, 0, 0):
                        blocks.append((2, (0, 0, 0)))
                else:
                    blocks.append((3, (bx, by, bz)))
    nb = len(blocks)
    info = [(i, lv, idx, 2.0 ** -lv / 8) for i, (lv, idx) in enumerate(blocks)]
    rows = nb * LAB_GHOSTS
    csr = {"row_ptr": np.arange(rows + 1, dtype=np.int64), "src": np.zeros(rows, dtype=np.int64),
           "w0": np.ones(rows), "w1": np.ones(rows), "w2": np.ones(rows)}
    return info, csr


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("gpd", [32, 64, 128])
def test_uq_dump_matches_oracle(gbfk_lib, prec, gpd):
    from gliomasolver_b200 import BlockPool

    R = np.float64 if prec == "f64" else np.float32
    info, csr = _mixed_level_blocks()
    nb = len(info)
    phi = np.random.default_rng(1).random(nb * 512).astype(R)
    want = O.uq_dump([b[1] for b in info], [b[2] for b in info], [b[3] for b in info], phi, gpd)
    with BlockPool(nb, prec) as pool:
        pool.set_topology(info, csr)
        pool.upload("phi", phi)
        got = pool.uq_dump(gpd)
    assert np.array_equal(got, want)


@pytest.mark.gpu
@pytest.mark.parametrize("use_roi", [False, True])
@pytest.mark.parametrize("use_pet", [False, True])
def test_log_likelihood_matches_oracle(gbfk_lib, use_roi, use_pet):
    from gliomasolver_b200 import BlockPool

    n = 32
    pw, pg, model, t1, fl, pet, roi = _observations(n, 5)
    r = roi if use_roi else None
    p = pet if use_pet else None
    want = O.log_likelihood(model, t1, fl, p, roi=r, step_pet=3, step_mri=2, **PARAMS)
    with BlockPool((n // 8) ** 3, "f64") as pool:
        pool.set_uniform(n // 8)
        pool.upload_dense("p_w", pw)
        pool.upload_dense("p_g", pg)
        pool.upload_dense("phi", model)
        assert np.array_equal(pool.uq_dump(n), model)
        pool.set_observations(t1, fl, p, r)
        got = pool.log_likelihood(step_pet=3, step_mri=2, **PARAMS)
    assert np.allclose(got[:3], want, rtol=1e-12, atol=1e-9)
    assert got[3] == pytest.approx(got[:3].sum(), rel=1e-15)
