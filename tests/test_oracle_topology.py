"""The oracle's adaptive-grid functions pinned to the reference: the RD
right-hand side through the ghost lists (fill_ghosts + rd_rhs_pool), per-block
wavelet details (fwt_detail_pool), block split (split_block) and collapse
(collapse_blocks) on an adapted grid with coarse-fine ghosts and a ball of CSF,
bit for bit against the reference's own ReactionDiffusionOperator sweep,
BlockFWT, Grid::refine and Grid::compress
(oracle/topo_harness.cpp): from the committed fixtures
(tests/golden/make_golden_topology.py) and, where the harness is built, live
on a larger grid for all three fields.  CPU only."""
import hashlib
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = Path(__file__).resolve().parent / "golden"
REALS = {"f64": np.float64, "f32": np.float32}


def _csr(row_ptr, src, w0, w1, w2):
    return {"row_ptr": np.ascontiguousarray(row_ptr, dtype=np.int64), "src": np.ascontiguousarray(src, dtype=np.int64),
            "w0": np.ascontiguousarray(w0), "w1": np.ascontiguousarray(w1), "w2": np.ascontiguousarray(w2)}


def _rhs(csr, fields, h, coeffs, R):
    pw, pg, phi = (fields[k].astype(R) for k in ("p_w", "p_g", "phi"))
    ghosts = [O.fill_ghosts(csr, a) for a in (pw, pg, phi)]
    assert np.any(pw + pg == 0)                      # no-flux cells present
    return O.rd_rhs_pool(h.astype(R), pw, pg, phi, *ghosts, *(R(c) for c in coeffs))


def _check(csr, fields, detail, parents, kids, collapsed, parent_fields, R):
    """fields / kids / parent_fields: {name: array} in float64 holding Real values."""
    nb = csr["row_ptr"].size - 1
    assert nb % 488 == 0
    nb //= 488
    phi = fields["phi"].astype(R)
    got = O.fwt_detail_pool(phi, O.fill_ghosts(csr, phi))
    assert np.array_equal(got, detail)
    assert detail.max() > 0
    for name, src in fields.items():
        src = src.astype(R)
        ghosts = O.fill_ghosts(csr, src).reshape(nb, 488)
        children = kids[name].reshape(-1, 8, 512).astype(R)
        for j, p in enumerate(parents):
            want = O.split_block(src.reshape(nb, 512)[p].copy(), ghosts[p].copy()).reshape(8, 512)
            assert np.array_equal(want, children[j]), (name, int(p))
        back = parent_fields[name].reshape(-1, 512).astype(R)
        for j, q in enumerate(collapsed):
            assert np.array_equal(O.collapse_blocks(children[q].ravel().copy()), back[j]), (name, int(q))


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_topology_functions_match_the_reference_fixture(prec):
    g = np.load(GOLDEN / f"topology_adapt_{prec}.npz")
    row_ptr = np.concatenate([[0], np.cumsum(g["row_len"].astype(np.int64))])
    src = np.cumsum(g["src_delta"].astype(np.int64))
    csr = _csr(row_ptr, src, g["w0"], g["w1"], g["w2"])
    # the grid has two levels, and some ghosts are interpolated across them
    assert len(set(g["level"].tolist())) == 2 and row_ptr[-1] > row_ptr.size - 1
    assert g["split_parent"].size == 8 and g["collapse_parent"].size > 0
    R = REALS[prec]
    rhs = _rhs(csr, {k: g[k] for k in ("p_w", "p_g", "phi")}, g["h"], g["coeffs"], R)
    assert np.array_equal(rhs.astype(np.float64)[::997], g["rhs_sample"])
    assert hashlib.sha256(rhs.tobytes()).digest() == g["rhs_sha256"].tobytes()
    _check(csr, {"phi": g["phi"]}, g["detail"], g["split_parent"], {"phi": g["split_phi"]}, g["collapse_parent"],
           {"phi": g["collapse_phi"]}, REALS[prec])


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_topology_functions_match_the_reference_live(prec):
    if not O.ref_topology_available(prec):
        pytest.skip("oracle/_ref/topo_harness is built only where the reference sources are")
    d = O.ref_topology(2, 5, 2e-2, 5, precision=prec)
    assert len(set(d["level"].tolist())) >= 3 and d["summary"]["split"] > 8
    names = ("p_w", "p_g", "phi")
    csr = _csr(d["row_ptr"], d["src"], d["w0"], d["w1"], d["w2"])
    rhs = _rhs(csr, d, d["h"], d["coeffs"], REALS[prec])
    assert np.array_equal(rhs, d["rhs"].astype(REALS[prec])) and np.abs(rhs).max() > 0
    _check(csr, {n: d[n] for n in names}, d["detail"],
           d["split_parent"], {n: d["split_" + n] for n in names}, d["collapse_parent"],
           {n: d["collapse_" + n] for n in names}, REALS[prec])
