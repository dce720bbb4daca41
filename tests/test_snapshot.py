"""Host snapshots of a block pool (gliomasolver_b200/snapshot.py): the file
round trip against a numpy stand-in of the pool's public calls (CPU), and on
the GPU a run that is saved, restored into a new pool and continued, bit for
bit equal to the run that was never interrupted, on a uniform grid and on a
ghost-list topology with permuted slots."""
import numpy as np
import pytest

from gliomasolver_b200.snapshot import FIELD_NAMES, load_snapshot, restore_pool, save_snapshot


class FakePool:
    """The calls snapshot.py uses, on numpy arrays."""

    def __init__(self, max_blocks, precision):
        self.max_blocks, self.precision = max_blocks, precision
        self.dtype = np.float64 if precision == "f64" else np.float32
        self.n = None
        self.mem = {f: np.zeros(max_blocks * 512, self.dtype) for f in FIELD_NAMES}
        self.topology = None

    def set_uniform(self, bpd):
        self.n, self.topology = 8 * bpd, ("uniform", bpd)

    def set_topology(self, blocks, csr):
        self.n, self.topology = None, ("lists", blocks, csr)

    def upload(self, field, values, first_cell=0):
        a = np.ascontiguousarray(values, dtype=self.dtype).ravel()
        self.mem[field][first_cell:first_cell + a.size] = a

    def download(self, field, ncells, first_cell=0):
        return self.mem[field][first_cell:first_cell + ncells].copy()


def _filled(pool, rng, nslots):
    for f in FIELD_NAMES:
        pool.upload(f, rng.random(nslots * 512))


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_uniform_round_trip(tmp_path, prec):
    rng = np.random.default_rng(0)
    a = FakePool(20, prec)
    a.set_uniform(2)
    _filled(a, rng, 8)
    save_snapshot(tmp_path / "s.npz", a, meta={"step": 17, "t": 3.25})
    assert sorted(p.name for p in tmp_path.iterdir()) == ["s.npz"]
    snap = load_snapshot(tmp_path / "s.npz")
    assert (snap.precision, snap.max_blocks, snap.blocks_per_dim, snap.meta) == (prec, 20, 2, {"step": 17, "t": 3.25})
    b = restore_pool(snap, pool=FakePool(20, prec))
    assert b.topology == ("uniform", 2)
    for f in FIELD_NAMES:
        assert np.array_equal(b.mem[f][:8 * 512], a.mem[f][:8 * 512])
        assert b.mem[f].dtype == a.dtype


def test_ghost_list_round_trip(tmp_path):
    rng = np.random.default_rng(1)
    blocks = [(5, 3, (1, 2, 3), 2.0 ** -6), (0, 3, (0, 0, 0), 2.0 ** -6), (9, 4, (7, 1, 0), 2.0 ** -7)]
    nrows = len(blocks) * 488
    csr = {"row_ptr": np.arange(nrows + 1, dtype=np.int64), "src": rng.integers(0, 10 * 512, nrows),
           "w0": rng.random(nrows), "w1": rng.random(nrows), "w2": np.ones(nrows)}
    a = FakePool(12, "f32")
    a.set_topology(blocks, csr)
    _filled(a, rng, 10)
    with pytest.raises(ValueError):
        save_snapshot(tmp_path / "s.npz", a)            # the pool keeps no host copy of the lists
    save_snapshot(tmp_path / "s.npz", a, topology=(blocks, csr))
    snap = load_snapshot(tmp_path / "s.npz")
    assert snap.blocks_per_dim is None and snap.blocks == blocks
    for k in csr:
        assert np.array_equal(snap.csr[k], csr[k])
    b = restore_pool(snap, pool=FakePool(12, "f32"))
    assert b.topology[0] == "lists" and b.topology[1] == blocks
    for f in FIELD_NAMES:
        assert np.array_equal(b.mem[f][:10 * 512], a.mem[f][:10 * 512])
    with pytest.raises(ValueError):
        restore_pool(snap, pool=FakePool(12, "f64"))
    with pytest.raises(ValueError):
        restore_pool(snap, pool=FakePool(9, "f32"))


def test_rejects_a_foreign_file(tmp_path):
    np.savez(tmp_path / "x.npz", header=np.frombuffer(b'{"format": 99}', dtype=np.uint8))
    with pytest.raises(ValueError):
        load_snapshot(tmp_path / "x.npz")


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_resumed_run_equals_the_uninterrupted_run(gbfk_lib, tmp_path, prec):
    from gliomasolver_b200 import BlockPool
    from gliomasolver_b200.anatomy import make_case
    from gliomasolver_b200.schedule import make_schedule

    n, bpd = 32, 4
    pw, pg, c0, _ = make_case(n, 0)
    s = make_schedule(0.13, 0.025, 150.0, 25.6, bpd, prec)
    with BlockPool(bpd ** 3, prec) as a:
        a.set_uniform(bpd)
        for name, v in (("p_w", pw), ("p_g", pg), ("phi", c0)):
            a.upload_dense(name, v)
        a.rd_step(s.Dw, s.Dg, s.rho, s.dt, 20)
        save_snapshot(tmp_path / "run.npz", a, meta={"step": 20})
        a.rd_step(s.Dw, s.Dg, s.rho, s.dt, 30)
        want = a.download_dense("phi")
    snap = load_snapshot(tmp_path / "run.npz")
    with restore_pool(snap) as b:
        b.rd_step(s.Dw, s.Dg, s.rho, s.dt, 50 - snap.meta["step"])
        got = b.download_dense("phi")
    assert np.array_equal(got, want)
    assert np.abs(want - c0.astype(want.dtype)).max() > 0


@pytest.mark.gpu
def test_resumed_ghost_list_run_equals_the_uninterrupted_run(gbfk_lib, tmp_path):
    from gliomasolver_b200 import BlockPool
    from gliomasolver_b200.anatomy import make_case
    from gliomasolver_b200.schedule import make_schedule
    from topology_util import dense_to_pool, uniform_topology

    n, bpd = 32, 4
    slots = np.random.default_rng(2).permutation(bpd ** 3 + 6)[: bpd ** 3]
    pw, pg, c0, _ = make_case(n, 3)
    blocks, csr = uniform_topology(bpd, slots)
    s = make_schedule(0.3, 0.1, 150.0, 25.6, bpd, "f64")
    ncells = (int(slots.max()) + 1) * 512
    with BlockPool(bpd ** 3 + 6, "f64") as a:
        a.set_topology(blocks, csr)
        for name, v in (("p_w", pw), ("p_g", pg), ("phi", c0)):
            a.upload(name, dense_to_pool(v, slots))
        a.rd_step(s.Dw, s.Dg, s.rho, s.dt, 7)
        save_snapshot(tmp_path / "run.npz", a, topology=(blocks, csr), meta={"step": 7})
        a.rd_step(s.Dw, s.Dg, s.rho, s.dt, 9)
        want = a.download("phi", ncells)
    with restore_pool(load_snapshot(tmp_path / "run.npz")) as b:
        b.rd_step(s.Dw, s.Dg, s.rho, s.dt, 9)
        got = b.download("phi", ncells)
    assert np.array_equal(got, want)
