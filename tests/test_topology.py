"""Block-pool topologies given as ghost lists (gbfk_set_topology): arbitrary
pool slots, faces that go through the ghost fill, wavelet details and
split/collapse, against the oracle."""
import numpy as np
import pytest

from gliomasolver_b200.anatomy import make_case
from gliomasolver_b200.schedule import make_schedule
from oracle import oracle as O
from topology_util import LAB_GHOSTS, dense_to_pool, face_rows, pool_to_dense, uniform_topology


def _pool_inputs(n, seed, R, slots):
    pw, pg, c0, _ = make_case(n, seed)
    pw, pg, c0 = (a.astype(R) for a in (pw, pg, c0))
    return pw, pg, c0, [dense_to_pool(a, slots) for a in (pw, pg, c0)]


def _oracle_pool_rhs(blocks, csr, pwp, pgp, php, s):
    order = np.array([b[0] for b in blocks])
    R = pwp.dtype.type
    pw_b, pg_b, ph_b = (a.reshape(-1, 512)[order].ravel() for a in (pwp, pgp, php))
    # ghost sources are pool cells: fill from the pool arrays
    gpw, gpg, gph = (O.fill_ghosts(csr, a) for a in (pwp, pgp, php))
    h = np.array([b[3] for b in blocks], dtype=R)
    return O.rd_rhs_pool(h, pw_b, pg_b, ph_b, gpw, gpg, gph, s.Dw, s.Dg, s.rho)


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_oracle_pool_path_equals_dense(prec):
    """The oracle's ghost-list path reproduces its dense periodic path (CPU)."""
    R = np.float64 if prec == "f64" else np.float32
    n, bpd = 16, 2
    slots = np.random.default_rng(0).permutation(bpd ** 3) + 3
    pw, pg, c0, (pwp, pgp, php) = _pool_inputs(n, 4, R, slots)
    blocks, csr = uniform_topology(bpd, slots, padded_rows=face_rows(1, 0))
    s = make_schedule(0.13, 0.025, 150.0, 25.6, bpd, prec)
    rhs_pool = _oracle_pool_rhs(blocks, csr, pwp, pgp, php, s)
    dense = O.rd_rhs_dense(pw, pg, c0, s.Dw, s.Dg, s.rho, s.h)
    bl = dense.reshape(bpd, 8, bpd, 8, bpd, 8).transpose(0, 2, 4, 1, 3, 5).reshape(-1)
    assert np.array_equal(rhs_pool, bl)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_ghost_list_topology_matches_uniform(gbfk_lib, prec):
    """Permuted slots and faces through the ghost fill give the same steps."""
    from gliomasolver_b200 import BlockPool

    R = np.float64 if prec == "f64" else np.float32
    n, bpd, steps = 32, 4, 12
    rng = np.random.default_rng(1)
    slots = rng.permutation(bpd ** 3 + 10)[: bpd ** 3]
    pw, pg, c0, (pwp, pgp, php) = _pool_inputs(n, 3, R, slots)
    padded = np.concatenate([face_rows(b, f) for b, f in ((0, 0), (5, 3), (17, 4), (63, 1))])
    blocks, csr = uniform_topology(bpd, slots, padded_rows=padded)
    s = make_schedule(0.3, 0.1, 150.0, 25.6, bpd, prec)
    want = O.rd_steps_dense(pw, pg, c0, s.Dw, s.Dg, s.rho, s.h, s.dt, steps)
    with BlockPool(bpd ** 3 + 10, prec) as pool:
        pool.set_topology(blocks, csr)
        for name, a in (("p_w", pwp), ("p_g", pgp), ("phi", php)):
            pool.upload(name, a)
        pool.rd_step(s.Dw, s.Dg, s.rho, s.dt, steps, check_nan=True)
        got = pool.download("phi", pwp.size)
    assert np.array_equal(pool_to_dense(got, slots, n), want)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_fwt_details_match_oracle(gbfk_lib, prec):
    from gliomasolver_b200 import BlockPool

    R = np.float64 if prec == "f64" else np.float32
    n, bpd = 32, 4
    slots = np.arange(bpd ** 3)[::-1].copy()
    pw, pg, c0, (pwp, pgp, php) = _pool_inputs(n, 5, R, slots)
    blocks, csr = uniform_topology(bpd, slots)
    order = np.array([b[0] for b in blocks])
    want = O.fwt_detail_pool(php.reshape(-1, 512)[order].ravel(), O.fill_ghosts(csr, php))
    with BlockPool(bpd ** 3, prec) as pool:
        pool.set_topology(blocks, csr)
        for name, a in (("p_w", pwp), ("p_g", pgp), ("phi", php)):
            pool.upload(name, a)
        got = pool.fwt_details()
    assert np.array_equal(got, want)
    assert want.max() > 0


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_split_and_collapse_match_oracle(gbfk_lib, prec):
    from gliomasolver_b200 import BlockPool

    R = np.float64 if prec == "f64" else np.float32
    n, bpd = 16, 2
    slots = np.arange(bpd ** 3)
    pw, pg, c0, (pwp, pgp, php) = _pool_inputs(n, 6, R, slots)
    blocks, csr = uniform_topology(bpd, slots)
    parents = np.array([0, 5])
    children = np.arange(8, 24).reshape(2, 8)
    with BlockPool(32, prec) as pool:
        pool.set_topology(blocks, csr)
        for name, a in (("p_w", pwp), ("p_g", pgp), ("phi", php)):
            pool.upload(name, np.concatenate([a, np.zeros(24 * 512 - a.size, R)]))
        pool.split(parents, children)
        fields = {f: pool.download(f, 32 * 512).reshape(32, 512) for f in ("phi", "p_w", "p_g")}
        # collapse the children of block 5 into slot 30
        pool.collapse(children[1:], [30])
        back = {f: pool.download(f, 32 * 512).reshape(32, 512)[30] for f in ("phi", "p_w", "p_g")}
    for f, src in (("phi", php), ("p_w", pwp), ("p_g", pgp)):
        g = O.fill_ghosts(csr, src).reshape(-1, LAB_GHOSTS)
        for i, b in enumerate(parents):
            want = O.split_block(src.reshape(-1, 512)[b].copy(), g[b].copy()).reshape(8, 512)
            assert np.array_equal(fields[f][children[i]], want), (f, b)
        want_parent = O.collapse_blocks(fields[f][children[1]].ravel().copy())
        assert np.array_equal(back[f], want_parent)
        # injection of an interpolated block returns the parent's own values
        assert np.array_equal(back[f], src.reshape(-1, 512)[5])


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_cfl_step_on_the_device(gbfk_lib, prec):
    """gbfk_cfl: the reference's dt formula at the finest leaf spacing (the
    schedule's dt on a uniform grid, bit for bit) and the largest local
    diffusion coefficient, against numpy in the same Real."""
    from gliomasolver_b200 import BlockPool

    R = np.float64 if prec == "f64" else np.float32
    n, bpd = 32, 4
    rng = np.random.default_rng(3)
    slots = rng.permutation(bpd ** 3 + 6)[: bpd ** 3]
    pw, pg, c0, (pwp, pgp, php) = _pool_inputs(n, 3, R, slots)
    s = make_schedule(0.3, 0.1, 150.0, 25.6, bpd, prec)
    want_d = (R(pw) * R(s.Dw) + R(pg) * R(s.Dg)).astype(R).max()
    blocks, csr = uniform_topology(bpd, slots)
    with BlockPool(bpd ** 3 + 6, prec) as pool:
        pool.set_topology(blocks, csr)
        pool.upload("p_w", pwp)
        pool.upload("p_g", pgp)
        c = pool.cfl(s.Dw, s.Dg)
        assert c["dt"] == s.dt and c["h_min"] == float(R(1.0 / n))
        assert c["max_diffusion"] == float(want_d)
        # a refined block: the step follows the finest spacing
        blocks[5] = (blocks[5][0], 1, blocks[5][2], 0.5 / n)
        pool.set_topology(blocks, csr)
        pool.upload("p_w", pwp)
        pool.upload("p_g", pgp)
        c = pool.cfl(s.Dw, s.Dg)
        h = R(0.5 / n)
        mx = max(R(s.Dw), R(s.Dg))
        assert c["h_min"] == float(h)
        assert c["dt"] == float(R(0.99 * np.float64(h) * np.float64(h) / (6.0 * np.float64(mx))))
