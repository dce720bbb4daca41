"""gbfk_rd_step_static: the allocation-free step, for callers that cannot let
the library call cudaMalloc (their device memory belongs to another allocator,
or their time loop must not pay cudaMalloc's device-wide synchronisation).

It is called through the C ABI on device buffers the test owns, twice in a
row (phi0 -> phi1 -> phi2), and each result must equal the context-based
entry point gbfk_rd_step bit for bit, the tolerance of every RD parity test
here.  This file sorts last so that a run stopping at the first failure has
already run every other test."""
import ctypes

import numpy as np
import pytest

from gliomasolver_b200 import BlockPool
from gliomasolver_b200 import _lib
from gliomasolver_b200.anatomy import make_case
from gliomasolver_b200.schedule import make_schedule

pytestmark = pytest.mark.gpu


def _pool_order(vol):
    n = vol.shape[0]
    bpd = n // 8
    return np.ascontiguousarray(vol.reshape(bpd, 8, bpd, 8, bpd, 8).transpose(0, 2, 4, 1, 3, 5).reshape(-1))


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("n", [32, 64])
def test_static_step_matches_rd_step_twice(gbfk_lib, prec, n):
    import torch

    R = np.float64 if prec == "f64" else np.float32
    tdt = torch.float64 if prec == "f64" else torch.float32
    pw, pg, c0, _ = make_case(n, 9)
    pw, pg, c0 = (a.astype(R) for a in (pw, pg, c0))
    s = make_schedule(0.2, 0.05, 300.0, 25.6, n // 8, prec)

    # the existing entry point: two steps, one at a time
    want = []
    with BlockPool((n // 8) ** 3, prec) as pool:
        pool.set_uniform(n // 8)
        pool.upload_dense("p_w", pw)
        pool.upload_dense("p_g", pg)
        pool.upload_dense("phi", c0)
        for _ in range(2):
            pool.rd_step(s.Dw, s.Dg, s.rho, s.dt, 1)
            want.append(_pool_order(pool.download_dense("phi")))

    dev = torch.device("cuda", 0)
    d_pw, d_pg, d_a = (torch.from_numpy(_pool_order(a)).to(dev) for a in (pw, pg, c0))
    d_b = torch.empty_like(d_a)
    stream = torch.cuda.current_stream(dev).cuda_stream
    L = _lib.load()
    code = _lib.GBFK_F64 if prec == "f64" else _lib.GBFK_F32
    got = []
    src, dst = d_a, d_b
    for _ in range(2):
        rc = L.gbfk_rd_step_static(code, n // 8, ctypes.c_void_p(d_pw.data_ptr()), ctypes.c_void_p(d_pg.data_ptr()),
                                   ctypes.c_void_p(src.data_ptr()), ctypes.c_void_p(dst.data_ptr()),
                                   s.Dw, s.Dg, s.rho, s.dt, ctypes.c_void_p(stream), 0)
        assert rc == _lib.GBFK_OK
        torch.cuda.synchronize(dev)
        got.append(dst.cpu().numpy().astype(R))
        src, dst = dst, src
    for g, w in zip(got, want):
        assert g.dtype == w.dtype
        assert np.array_equal(g, w)
    assert not np.array_equal(got[0], got[1])


def test_static_step_rejects_grids_beyond_its_scratch(gbfk_lib):
    import torch

    L = _lib.load()
    dev = torch.device("cuda", 0)
    buf = torch.zeros(16, device=dev)
    p = ctypes.c_void_p(buf.data_ptr())
    q = ctypes.c_void_p(buf[8:].data_ptr())
    # 9^3 = 729 blocks > 512: refused before any device work
    assert L.gbfk_rd_step_static(_lib.GBFK_F32, 9, p, p, p, q, 1e-4, 1e-5, 0.1, 0.1, None, 0) == 7
    # the input and the output must differ
    assert L.gbfk_rd_step_static(_lib.GBFK_F32, 2, p, p, p, p, 1e-4, 1e-5, 0.1, 0.1, None, 0) == 1


def test_static_step_argument_checks(gbfk_lib):
    """Overlapping input and output ranges and a stream of another device are
    refused before any device work; the caller's current device is kept."""
    import torch

    L = _lib.load()
    dev = torch.device("cuda", 0)
    n = 2 * 2 * 2 * 512
    buf = torch.zeros(3 * n, device=dev)
    at = lambda k: ctypes.c_void_p(buf[k:].data_ptr())  # noqa: E731
    # phi_out starts inside phi_in (an offset into the same allocation)
    assert L.gbfk_rd_step_static(_lib.GBFK_F32, 2, at(0), at(0), at(0), at(n - 1), 1e-4, 1e-5, 0.1, 0.1, None, 0) == 1
    assert L.gbfk_rd_step_static(_lib.GBFK_F32, 2, at(0), at(0), at(n - 1), at(0), 1e-4, 1e-5, 0.1, 0.1, None, 0) == 1
    # adjacent ranges do not overlap
    torch.cuda.set_device(0)
    assert L.gbfk_rd_step_static(_lib.GBFK_F32, 2, at(0), at(0), at(0), at(n), 1e-4, 1e-5, 0.1, 0.1, None, 0) == 0
    torch.cuda.synchronize(dev)
    assert torch.cuda.current_device() == 0
    if torch.cuda.device_count() > 1:
        other = torch.cuda.Stream(device=1)
        assert L.gbfk_rd_step_static(_lib.GBFK_F32, 2, at(0), at(0), at(0), at(n), 1e-4, 1e-5, 0.1, 0.1,
                                     ctypes.c_void_p(other.cuda_stream), 0) == 1
