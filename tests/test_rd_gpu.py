"""Parity of the fused sm_100a RD step with the oracle, through the C ABI.

The bar is bit-exactness for both Real types: the device kernel performs the
reference's operations in the reference's order with the reference's
rounding (gbfk_exact.cuh), so its output must equal the reference's output
(the golden fixtures, made by the reference's own code) and the oracle's
output bit for bit.  At the benchmark size (256^3) the oracle is run for a
few steps on the CPU.
"""
import hashlib

import numpy as np
import pytest

from gliomasolver_b200 import BlockPool, BlockProcessing, GbfkError, reaction_diffusion_step
from gliomasolver_b200.anatomy import make_case
from gliomasolver_b200.schedule import make_schedule
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


def _fixture_inputs(fx):
    n, seed, prec = int(fx["n"]), int(fx["seed"]), str(fx["precision"])
    R = np.float64 if prec == "f64" else np.float32
    pw, pg, c0, _ = make_case(n, seed)
    pw, pg, c0 = (a.astype(R) for a in (pw, pg, c0))
    h = hashlib.sha256()
    for a in (pw, pg, c0):
        h.update(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    assert h.hexdigest() == str(fx["input_sha"])
    return n, prec, pw, pg, c0


def _pool(n, prec, pw, pg, c0):
    pool = BlockPool((n // 8) ** 3, prec)
    pool.set_uniform(n // 8)
    pool.upload_dense("p_w", pw)
    pool.upload_dense("p_g", pg)
    pool.upload_dense("phi", c0)
    return pool


@pytest.mark.parametrize("name", ["rhs_n32_f64", "rhs_n32_f32"])
def test_rhs_bit_exact_vs_reference(gbfk_lib, golden, name):
    fx = golden(name)
    n, prec, pw, pg, c0 = _fixture_inputs(fx)
    with _pool(n, prec, pw, pg, c0) as pool:
        rhs = pool.rd_rhs(fx["Dw"], fx["Dg"], fx["rho"])
    # pool order -> dense
    bpd = n // 8
    dense = rhs.reshape(bpd, bpd, bpd, 8, 8, 8).transpose(0, 3, 1, 4, 2, 5).reshape(n, n, n)
    assert np.array_equal(dense.astype(np.float64), fx["out"])


@pytest.mark.parametrize("name", ["steps_n32_f64", "steps_n32_f32", "steps_n16_f64_fast"])
def test_steps_bit_exact_vs_reference(gbfk_lib, golden, name):
    fx = golden(name)
    n, prec, pw, pg, c0 = _fixture_inputs(fx)
    with _pool(n, prec, pw, pg, c0) as pool:
        pool.rd_step(fx["Dw"], fx["Dg"], fx["rho"], fx["dt"], int(fx["nsteps"]), check_nan=True)
        out = pool.download_dense("phi")
    assert np.array_equal(out.astype(np.float64), fx["out"])


def test_config1_full_run_bit_exact(gbfk_lib, golden):
    """The parity configuration: 64^3, FP64, 739 steps to T = 150 d."""
    fx = golden("config1_n64_f64")
    n, prec, pw, pg, c0 = _fixture_inputs(fx)
    with _pool(n, prec, pw, pg, c0) as pool:
        pool.rd_step(fx["Dw"], fx["Dg"], fx["rho"], fx["dt"], int(fx["nsteps"]), check_nan=True)
        out = pool.download_dense("phi")
    sub = out[::4, ::4, ::4].astype(np.float64)
    rel = np.linalg.norm(sub - fx["out_sub"]) / np.linalg.norm(fx["out_sub"])
    assert rel <= 1e-12
    assert _sha(out) == str(fx["output_sha"])


def test_operator_interface_matches_direct_call(gbfk_lib):
    """BlockProcessing.pipeline_process + process == gbfk_rd_step."""
    n = 16
    pw, pg, c0, _ = make_case(n, 2)
    s = make_schedule(0.13, 0.025, 150.0, 25.6, n // 8, "f64")
    with _pool(n, "f64", pw, pg, c0) as a, _pool(n, "f64", pw, pg, c0) as b:
        bp = BlockProcessing()
        for _ in range(5):
            reaction_diffusion_step(a, s.Dw, s.Dg, s.rho, s.dt, bp)
        b.rd_step(s.Dw, s.Dg, s.rho, s.dt, 5)
        assert np.array_equal(a.download_dense("phi"), b.download_dense("phi"))
        with pytest.raises(GbfkError):
            BlockProcessing().process(None, a, __import__("gliomasolver_b200").UpdateTumor(s.dt))


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("n,seed,steps", [(8, 4, 9), (16, 6, 21), (48, 8, 6)])
def test_edge_cases_vs_oracle(gbfk_lib, prec, n, seed, steps):
    """One block that is its own periodic neighbour (n = 8), CSF holes next to
    tumour, values above 1 (clamp), cells with no tissue but tumour, an empty
    tissue slab, and a non-power-of-two block count."""
    R = np.float64 if prec == "f64" else np.float32
    pw, pg, c0, _ = make_case(n, seed)
    rng = np.random.default_rng(seed)
    c0 = np.maximum(c0, rng.uniform(0, 1, c0.shape) * (rng.uniform(0, 1, c0.shape) < 0.05))
    c0[0, 0, :] = 1.7
    pw[n // 2, :, : n // 3] = 0.0
    pg[n // 2, :, : n // 3] = 0.0
    pw[:, 1, :] = 0.0
    pg[:, 1, :] = 0.0
    pw, pg, c0 = (a.astype(R) for a in (pw, pg, c0))
    s = make_schedule(0.3, 0.2, 300.0, 25.6, n // 8, prec)
    want = O.rd_steps_dense(pw, pg, c0, s.Dw, s.Dg, s.rho, s.h, s.dt, steps)
    with _pool(n, prec, pw, pg, c0) as pool:
        pool.rd_step(s.Dw, s.Dg, s.rho, s.dt, steps)
        got = pool.download_dense("phi")
    assert np.array_equal(got, want)


def test_no_tissue_reaction_only(gbfk_lib):
    """No tissue anywhere: cells with phi > 0 still count as inside the domain
    (p_w + p_g + phi > 0) and only react; cells with phi <= 0 are clamped."""
    n = 16
    pw = np.zeros((n, n, n))
    pg = np.zeros((n, n, n))
    c0 = np.linspace(-0.5, 1.5, n ** 3).reshape(n, n, n)
    want = O.rd_steps_dense(pw, pg, c0, 1e-3, 1e-4, 0.1, 1 / n, 0.5, 3)
    with _pool(n, "f64", pw, pg, c0) as pool:
        pool.rd_step(1e-3, 1e-4, 0.1, 0.5, 3)
        got = pool.download_dense("phi")
    assert np.array_equal(got, want)


def test_nan_is_reported(gbfk_lib):
    n = 8
    pw, pg, c0, _ = make_case(n, 1)
    c0[3, 3, 3] = np.nan
    with _pool(n, "f32", pw, pg, c0) as pool:
        with pytest.raises(GbfkError) as e:
            pool.rd_step(1e-3, 1e-4, 0.1, 0.5, 1, check_nan=True)
        assert e.value.code == 4


def test_benchmark_size_f32_vs_oracle(gbfk_lib):
    """256^3 (32768 blocks), FP32 storage, 3 steps: bit-exact vs the oracle."""
    n = 256
    pw, pg, c0, _ = make_case(n, 0)
    pw, pg, c0 = (a.astype(np.float32) for a in (pw, pg, c0))
    s = make_schedule(0.2, 0.05, 300.0, 25.6, n // 8, "f32")
    want = O.rd_steps_dense(pw, pg, c0, s.Dw, s.Dg, s.rho, s.h, s.dt, 3)
    with _pool(n, "f32", pw, pg, c0) as pool:
        pool.rd_step(s.Dw, s.Dg, s.rho, s.dt, 3)
        got = pool.download_dense("phi")
    assert np.array_equal(got, want)


def test_fp32_storage_error_vs_fp64(gbfk_lib):
    """FP32 storage against the FP64 path after 200 steps at 128^3."""
    n = 128
    pw, pg, c0, _ = make_case(n, 0)
    s64 = make_schedule(0.2, 0.05, 300.0, 25.6, n // 8, "f64")
    s32 = make_schedule(0.2, 0.05, 300.0, 25.6, n // 8, "f32")
    with _pool(n, "f64", pw, pg, c0) as a, _pool(n, "f32", pw, pg, c0) as b:
        a.rd_step(s64.Dw, s64.Dg, s64.rho, s64.dt, 200)
        b.rd_step(s32.Dw, s32.Dg, s32.rho, s32.dt, 200)
        x, y = a.download_dense("phi"), b.download_dense("phi").astype(np.float64)
    rel = np.linalg.norm(x - y) / np.linalg.norm(x)
    assert rel <= 1e-5


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("n,seed,steps", [(8, 3, 7), (32, 2, 9), (64, 9, 5)])
def test_pipelined_step_equals_block_step(gbfk_lib, prec, n, seed, steps):
    """The persistent TMA-fed step and the one-CTA-per-block step on the same
    uniform power-of-two grid give bit-identical fields after every step, and
    both equal the oracle: with tumour outside the anatomy (empty blocks with
    cells inside the domain), negative values and values above 1."""
    R = np.float64 if prec == "f64" else np.float32
    pw, pg, c0, _ = make_case(n, seed)
    rng = np.random.default_rng(seed + 100)
    c0 = np.maximum(c0, rng.uniform(0, 1, c0.shape) * (rng.uniform(0, 1, c0.shape) < 0.03))
    c0[0, 0, :] = 1.7
    c0[1, :, 2] = -0.3
    pw[n // 2, :, : n // 3] = 0.0
    pg[n // 2, :, : n // 3] = 0.0
    pw, pg, c0 = (a.astype(R) for a in (pw, pg, c0))
    s = make_schedule(0.3, 0.2, 300.0, 25.6, n // 8, prec)
    with _pool(n, prec, pw, pg, c0) as a, _pool(n, prec, pw, pg, c0) as b:
        assert a.step_kernel == ""
        a.step_kernel = "pipelined"
        b.step_kernel = "block"
        for _ in range(steps):
            a.rd_step(s.Dw, s.Dg, s.rho, s.dt, 1, check_nan=True)
            b.rd_step(s.Dw, s.Dg, s.rho, s.dt, 1, check_nan=True)
            assert np.array_equal(a.download_dense("phi"), b.download_dense("phi"))
        assert a.step_kernel == "pipelined" and b.step_kernel == "block"
        got = a.download_dense("phi")
        # a field uploaded after steps (negative values again) takes the
        # pipeline's unclamped path once more
        for q in (a, b):
            q.upload_dense("phi", c0)
            q.rd_step(s.Dw, s.Dg, s.rho, s.dt, 2)
        assert np.array_equal(a.download_dense("phi"), b.download_dense("phi"))
    want = O.rd_steps_dense(pw, pg, c0, s.Dw, s.Dg, s.rho, s.h, s.dt, steps)
    assert np.array_equal(got, want)


def test_pipelined_step_kernel_selection(gbfk_lib):
    """AUTO picks the pipeline on uniform power-of-two grids and the block
    kernel elsewhere; forcing the pipeline where it does not apply is an
    error, and the pool stays usable."""
    pw, pg, c0, _ = make_case(48, 1)
    s = make_schedule(0.2, 0.05, 300.0, 25.6, 6, "f32")
    with _pool(48, "f32", *(a.astype(np.float32) for a in (pw, pg, c0))) as pool:
        pool.rd_step(s.Dw, s.Dg, s.rho, s.dt, 1)
        assert pool.step_kernel == "block"
        pool.step_kernel = "pipelined"
        with pytest.raises(GbfkError) as e:
            pool.rd_step(s.Dw, s.Dg, s.rho, s.dt, 1)
        assert e.value.code == 6
        pool.step_kernel = "auto"
        pool.rd_step(s.Dw, s.Dg, s.rho, s.dt, 1, check_nan=True)
    pw, pg, c0, _ = make_case(32, 1)
    with _pool(32, "f64", pw, pg, c0) as pool:
        pool.rd_step(1e-3, 1e-4, 0.1, 0.5, 2, check_nan=True)
        assert pool.step_kernel == "pipelined"
        # runs of steps in one launch on request
        pool.step_kernel = "run"
        pool.rd_step(1e-3, 1e-4, 0.1, 0.5, 3, check_nan=True)
        assert pool.step_kernel == "run"
        pool.sync()


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("n,seed,steps", [(8, 3, 7), (32, 2, 2), (64, 9, 3), (64, 5, 40), (128, 1, 101)])
def test_run_of_steps_equals_single_steps(gbfk_lib, prec, n, seed, steps):
    """A run of steps in one launch (grid barrier between steps) gives the
    bits of one pipelined launch per step: from an unclamped field (negative
    values, values above 1; the run starts after one single step), with
    tumour outside the anatomy (empty blocks whose cells read their
    neighbours from global memory every step), odd and even step counts."""
    R = np.float64 if prec == "f64" else np.float32
    pw, pg, c0, _ = make_case(n, seed)
    rng = np.random.default_rng(seed + 100)
    c0 = np.maximum(c0, rng.uniform(0, 1, c0.shape) * (rng.uniform(0, 1, c0.shape) < 0.03))
    c0[0, 0, :] = 1.7
    c0[1, :, 2] = -0.3
    pw[n // 2, :, : n // 3] = 0.0
    pg[n // 2, :, : n // 3] = 0.0
    pw, pg, c0 = (a.astype(R) for a in (pw, pg, c0))
    s = make_schedule(0.3, 0.2, 300.0, 25.6, n // 8, prec)
    with _pool(n, prec, pw, pg, c0) as a, _pool(n, prec, pw, pg, c0) as b:
        a.step_kernel = "run"
        b.step_kernel = "pipelined"
        a.rd_step(s.Dw, s.Dg, s.rho, s.dt, steps, check_nan=True)
        for _ in range(steps):
            b.rd_step(s.Dw, s.Dg, s.rho, s.dt, 1)
        # (two steps from an unclamped field are two single steps)
        assert a.step_kernel == ("run" if steps > 2 else "pipelined") and b.step_kernel == "pipelined"
        x = a.download_dense("phi")
        assert np.array_equal(x, b.download_dense("phi"))
        # a clamped field: the whole call is one run; twice in a row
        for _ in range(2):
            a.rd_step(s.Dw, s.Dg, s.rho, s.dt, steps, check_nan=True)
            for _ in range(steps):
                b.rd_step(s.Dw, s.Dg, s.rho, s.dt, 1)
            assert a.step_kernel == "run"
            assert np.array_equal(a.download_dense("phi"), b.download_dense("phi"))
    if n <= 32:
        want = O.rd_steps_dense(pw, pg, c0, s.Dw, s.Dg, s.rho, s.h, s.dt, steps)
        assert np.array_equal(x, want)


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_host_to_host_steps_equal_upload_step_download(gbfk_lib, prec):
    """gbfk_rd_step_host (asynchronous, two copy streams, two staging sets):
    five calls in a row from different initial states, each output equal to
    upload + gbfk_rd_step + download of the same state."""
    R = np.float64 if prec == "f64" else np.float32
    n = 32
    pw, pg, c0, _ = make_case(n, 4)
    s = make_schedule(0.2, 0.05, 150.0, 25.6, n // 8, prec)
    rng = np.random.default_rng(9)
    ins = [np.ascontiguousarray((c0 * rng.uniform(0.2, 1.0)).astype(R)) for _ in range(5)]
    steps = [1, 3, 0, 7, 2]
    with _pool(n, prec, pw.astype(R), pg.astype(R), ins[0]) as a, _pool(n, prec, pw.astype(R), pg.astype(R),
                                                                        ins[0]) as b:
        want = []
        for x, k in zip(ins, steps):
            b.upload_dense("phi", x)
            b.rd_step(s.Dw, s.Dg, s.rho, s.dt, k)
            want.append(b.download_dense("phi"))
        outs = [np.empty_like(x) for x in ins]
        for x, o, k in zip(ins, outs, steps):
            a.rd_step_host(x, o, s.Dw, s.Dg, s.rho, s.dt, k)
        a.sync()
        for i in range(5):
            assert np.array_equal(outs[i], want[i]), i
        assert np.array_equal(a.download_dense("phi"), want[-1])


def test_bounded_wait_gives_up_and_the_device_stays_usable(gbfk_lib):
    """Failure detection without a fault: a wait on an mbarrier phase that
    nothing completes (the bounded wait of the pipelined step) gives up after
    its 1 s limit and is reported as GBFK_E_TIMEOUT; the device keeps working."""
    import ctypes

    from gliomasolver_b200._lib import STATUS_CODES

    secs = ctypes.c_double(0)
    rc = gbfk_lib.gbfk_probe_bounded_wait(0, ctypes.byref(secs))
    assert rc == STATUS_CODES["GBFK_E_TIMEOUT"]
    assert 0.9 < secs.value < 10.0
    n = 16
    pw, pg, c0, _ = make_case(n, 2)
    s = make_schedule(0.13, 0.025, 150.0, 25.6, n // 8, "f64")
    with _pool(n, "f64", pw, pg, c0) as pool:
        pool.rd_step(s.Dw, s.Dg, s.rho, s.dt, 4, check_nan=True)
        got = pool.download_dense("phi")
    assert np.array_equal(got, O.rd_steps_dense(pw, pg, c0, s.Dw, s.Dg, s.rho, s.h, s.dt, 4))
