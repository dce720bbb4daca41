"""The oracle's UQ dump pinned to the reference's own
Glioma_ReactionDiffusion::_dumpUQoutput (oracle/uq_harness.cpp: the
reference's class after its _ic on a synthetic anatomy, adapted by its own
AutomaticRefinement / AutomaticCompression), bit for bit, on grids with blocks
finer than the dump grid, as fine, and 2, 4 and 8 times coarser.  The
reference allocates the dump without initialising it (Glioma/Matrix.h D3D),
so voxels that no block writes (blocks 8 times coarser) are compared only on
our side, where they are 0.  CPU only."""
import numpy as np
import pytest

from gliomasolver_b200.anatomy import make_case
from oracle import oracle as O

REALS = {"f64": np.float64, "f32": np.float32}
TUMOR = (0.5, 0.45, 0.55)
# (phi: 0 = the reference's own tumour ball, else a Gaussian of that width; refine tol; compress tol; levels)
CASES = [(0.0, 1e-3, 0.0, {3, 4}), (0.08, 1e-3, 0.0, {3, 4}), (0.08, 1e-2, 1e-3, {2, 3}),
         (0.08, 1e-2, 3e-2, {1, 2}), (0.08, 1e-3, 0.3, {0})]


@pytest.fixture(scope="module")
def anatomy(tmp_path_factory):
    d = tmp_path_factory.mktemp("uq")
    pw, pg, _, _ = make_case(64, 2)
    csf = ((pw + pg) == 0).astype(np.float64)
    for k, v in (("GM", pg), ("WM", pw), ("CSF", csf)):
        O.write_matrix3d(d / f"P_{k}.dat", v)
    return d / "P_"


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("sigma,rtol,ctol,levels", CASES)
def test_uq_dump_matches_the_reference(anatomy, prec, sigma, rtol, ctol, levels):
    if not O.ref_uq_available(prec):
        pytest.skip("oracle/_ref/uq_harness is built only where the reference sources are")
    R = REALS[prec]
    d = O.ref_uq_dump(anatomy, TUMOR, rtol, ctol, prec, sigma=sigma)
    assert set(int(v) for v in np.unique(d["level"])) == levels, d["summary"]
    gpd = d["summary"]["gpd"]
    lv, ix, h = d["level"], d["index"].reshape(-1, 3), d["h"].astype(R)
    got = O.uq_dump(lv, ix, h, d["phi"].astype(R), gpd)
    written = O.uq_dump(lv, ix, h, np.ones_like(d["phi"], dtype=R), gpd) != 0
    assert np.array_equal(got[written], d["dump"][written])
    assert np.all(got[~written] == 0)
    assert written.all() == (min(levels) > 0)
    assert np.abs(got).max() > 0.01
