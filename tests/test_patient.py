"""Patient data (gliomasolver_b200.patient over libgbfk's host functions):
Matrix files, the anatomy mapping of Glioma_ReactionDiffusion::_ic and the
likelihood inputs.

The mapping must give the reference's cells bit for bit: against the
golden fixture made by the reference's own _ic (tests/golden/
make_golden_anatomy.py), against the oracle's C restatement on volumes
with every branch of the mapping, and, where oracle/_ref is built, against
the reference directly.  These calls need no GPU.
"""
import os

import numpy as np
import pytest

from gliomasolver_b200 import patient
from gliomasolver_b200._lib import STATUS_CODES, GbfkError
from oracle import oracle as O

E_IO, E_INVALID = STATUS_CODES["GBFK_E_IO"], STATUS_CODES["GBFK_E_INVALID"]


@pytest.fixture(scope="module", autouse=True)
def _library():
    from gliomasolver_b200.build import build_library

    build_library()


# ----------------------------------------------------------------- Matrix files
def test_matrix_layout_matches_the_reference_format(tmp_path):
    rng = np.random.default_rng(0)
    v3 = rng.standard_normal((5, 4, 3))
    pts = np.array([[1, 2, 3], [4, 5, 6], [7, 8, 9], [0, 1, 2]], dtype=np.float64)
    O.write_matrix3d(tmp_path / "a.dat", v3)
    O.write_matrix2d(tmp_path / "roi.dat", pts)
    patient.write_matrix(tmp_path / "b.dat", v3)
    patient.write_matrix(tmp_path / "roi2.dat", pts.T)
    assert (tmp_path / "a.dat").read_bytes() == (tmp_path / "b.dat").read_bytes()
    assert (tmp_path / "roi.dat").read_bytes() == (tmp_path / "roi2.dat").read_bytes()
    info = patient.matrix_info(tmp_path / "a.dat")
    assert (info.dim, info.sizes, info.type_id) == (3, (3, 4, 5), 0)
    assert np.array_equal(patient.read_matrix(tmp_path / "a.dat"), v3)
    assert np.array_equal(patient.read_roi(tmp_path / "roi.dat"), pts.astype(np.int32))


@pytest.mark.parametrize("tid,dtype", [(0, np.float64), (1, np.float32), (2, np.int32)])
def test_matrix_type_ids_round_trip(tmp_path, tid, dtype):
    rng = np.random.default_rng(tid)
    v = rng.uniform(-1000, 1000, (3, 6, 7))
    patient.write_matrix(tmp_path / "m.dat", v, type_id=tid)
    raw = (tmp_path / "m.dat").read_bytes()
    head = np.frombuffer(raw[:24], dtype=np.int32)
    assert list(head) == [1234, 3, 7, 6, 3, tid]
    want = v.astype(dtype)                              # float rounds, int truncates towards zero
    assert np.array_equal(np.frombuffer(raw[24:], dtype=dtype).reshape(v.shape), want)
    assert np.array_equal(patient.read_matrix(tmp_path / "m.dat"), want.astype(np.float64))
    assert patient.matrix_info(tmp_path / "m.dat").type_id == tid


def test_matrix_errors(tmp_path):
    good = tmp_path / "g.dat"
    patient.write_matrix(good, np.ones((2, 2, 2)))
    raw = good.read_bytes()
    cases = {
        "missing.dat": None,
        "swapped.dat": np.array([1234], dtype=">i4").tobytes() + raw[4:],
        "dim4.dat": np.int32(1234).tobytes() + np.int32(4).tobytes() + raw[8:],
        "short.dat": raw[:-8],
        "header.dat": raw[:10],
        "tid.dat": raw[:20] + np.int32(3).tobytes() + raw[24:],
        "neg.dat": raw[:8] + np.int32(-2).tobytes() + raw[12:],
    }
    for name, data in cases.items():
        if data is not None:
            (tmp_path / name).write_bytes(data)
        with pytest.raises(GbfkError) as e:
            patient.read_matrix(tmp_path / name)
        assert e.value.code == E_IO, name
    with pytest.raises(GbfkError) as e:
        patient.write_matrix(tmp_path / "i.dat", np.array([[3e9, 1.0]]), type_id=2)
    assert e.value.code == E_INVALID
    with pytest.raises(GbfkError) as e:
        patient.write_matrix(tmp_path / "nodir" / "x.dat", np.ones((2, 2)))
    assert e.value.code == E_IO
    # reading into a buffer that is too small
    import ctypes

    from gliomasolver_b200 import _lib
    buf = np.empty(7)
    assert _lib.load().gbfk_matrix_read(os.fsencode(good), buf.ctypes.data_as(ctypes.c_void_p), 7) == E_INVALID


def test_empty_and_two_dimensional(tmp_path):
    patient.write_matrix(tmp_path / "e.dat", np.zeros((0, 4, 3)))
    assert patient.read_matrix(tmp_path / "e.dat").shape == (0, 4, 3)
    v = np.arange(12.0).reshape(3, 4)
    patient.write_matrix(tmp_path / "d2.dat", v, type_id=1)
    assert patient.matrix_info(tmp_path / "d2.dat").sizes == (4, 3)
    assert np.array_equal(patient.read_matrix(tmp_path / "d2.dat"), v)


# ------------------------------------------------------------ anatomy mapping
FIELDS = ("p_w", "p_g", "p_csf", "phi")


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_mapping_matches_the_reference_golden(golden, tmp_path, prec):
    g = golden("anatomy_ic")
    for k, v in (("GM", g["gm"]), ("WM", g["wm"]), ("CSF", g["csf"])):
        patient.write_matrix(tmp_path / f"P_{k}.dat", v)
    for bpd in (2, 3):
        a = patient.load_patient(tmp_path / "P_", bpd, g[f"tic_bpd{bpd}"], prec)
        for k in FIELDS:
            want = g[f"{prec}_bpd{bpd}_{k}"]
            got = getattr(a, k)
            assert got.dtype == want.dtype and np.array_equal(got, want), (bpd, k)
        assert a.L_cm == float(g[f"{prec}_bpd{bpd}_L"])


def _tricky_volumes(shape, seed):
    rng = np.random.default_rng(seed)
    gm, wm = rng.uniform(0, 1, shape), rng.uniform(0, 1, shape)
    csf = rng.uniform(0, 1, shape) ** 3
    m = rng.uniform(0, 1, shape)
    csf[m < 0.05] = (gm + wm)[m < 0.05]
    big = m > 0.95
    gm[big] *= 1.5
    wm[big] *= 1.5
    csf[big] = 2.5
    tiny = (m > 0.3) & (m < 0.33)
    gm[tiny], wm[tiny], csf[tiny] = 2e-4, 3e-4, 0.0
    zero = (m > 0.4) & (m < 0.42)
    gm[zero] = wm[zero] = csf[zero] = 0.0
    return gm, wm, csf


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("shape,bpd,tic", [((30, 41, 37), 4, (0.5, 0.45, 0.4)),
                                           ((64, 64, 64), 8, (0.3, 0.52, 0.61)),
                                           ((20, 27, 33), 3, (0.2, 0.3, 0.25)),
                                           ((9, 10, 11), 1, (0.0, 0.0, 0.0))])
def test_mapping_matches_the_oracle(prec, shape, bpd, tic):
    gm, wm, csf = _tricky_volumes(shape, bpd)
    a = patient.map_anatomy(gm, wm, csf, bpd, tic, prec)
    o = O.map_anatomy(gm, wm, csf, bpd, tic, prec)
    for k in FIELDS + ("tissue",):
        assert np.array_equal(getattr(a, k), o[k]), k
    assert a.L_cm == (max(shape) * 0.1 if prec == "f64" else float(np.float32(max(shape) * 0.1)))
    n = 8 * bpd
    assert a.phi.shape == (n, n, n) and a.phi.dtype == (np.float64 if prec == "f64" else np.float32)
    # the smoothed ball never reaches 1: its radius (0.005) is below its half-width (1/64)
    assert a.phi.max() < 1.0


def test_mapping_against_the_reference(tmp_path):
    """The reference's own _ic, where oracle/_ref is built (a 128^3 grid from a
    non-cubic volume, and a bpd that is not a power of two)."""
    if not O.ref_ic_available("f64") or not O.ref_ic_available("f32"):
        pytest.skip("oracle/_ref/ic_harness is built only where the reference sources are")
    for shape, bpd, tic in (((50, 60, 70), 16, (0.5, 0.5, 0.5)), ((20, 27, 33), 3, (0.2, 0.3, 0.25))):
        gm, wm, csf = _tricky_volumes(shape, 5)
        for k, v in (("GM", gm), ("WM", wm), ("CSF", csf)):
            patient.write_matrix(tmp_path / f"Q_{k}.dat", v)
        for prec in ("f64", "f32"):
            a = patient.load_patient(tmp_path / "Q_", bpd, tic, prec)
            r = O.ref_map_anatomy(tmp_path / "Q_", bpd, tic, prec)
            for k in FIELDS:
                assert np.array_equal(getattr(a, k).astype(np.float64), r[k]), (shape, prec, k)
            assert a.L_cm == r["L"]


def test_mapping_rejects_bad_arguments():
    v = np.ones((4, 4, 4))
    with pytest.raises(ValueError):
        patient.map_anatomy(v, v, np.ones((4, 4, 5)), 2, (0.5, 0.5, 0.5))
    with pytest.raises(GbfkError) as e:
        patient.map_anatomy(v, v, v, 0, (0.5, 0.5, 0.5))
    assert e.value.code == E_INVALID
    with pytest.raises(GbfkError):
        patient.map_anatomy(np.ones((0, 4, 4)), np.ones((0, 4, 4)), np.ones((0, 4, 4)), 2, (0.5, 0.5, 0.5))


# ------------------------------------------------------------ likelihood inputs
def test_load_observations(tmp_path):
    rng = np.random.default_rng(3)
    n = 16
    t1 = (rng.uniform(0, 1, (n, n, n)) > 0.7).astype(np.float64)
    fl = (rng.uniform(0, 1, (n, n, n)) > 0.5).astype(np.float64)
    pet = rng.uniform(0, 1, (n, n, n))
    pts = rng.integers(0, n, (25, 3)).astype(np.float64) + 0.75     # the reference truncates to int
    O.write_matrix3d(tmp_path / "tumT1c.dat", t1)
    O.write_matrix3d(tmp_path / "tumFLAIR.dat", fl)
    O.write_matrix3d(tmp_path / "tumPET.dat", pet)
    O.write_matrix2d(tmp_path / "ROI.dat", pts)
    (tmp_path / "LikelihoodInput.txt").write_text("0.000361 0.85\n0.7 0.25 2\n")
    (tmp_path / "TumorIC.txt").write_text("0.28 0.67 0.35\n")
    obs = patient.load_observations(tmp_path, roi=True)
    assert np.array_equal(obs.t1c, t1) and np.array_equal(obs.flair, fl) and np.array_equal(obs.pet, pet)
    assert obs.roi.dtype == np.int32 and np.array_equal(obs.roi, np.trunc(pts).astype(np.int32))
    assert obs.params == {"pet_sigma2": 0.000361, "pet_scale": 0.85, "t1_uc": 0.7, "t2_uc": 0.25, "slope": 2.0}
    assert obs.likelihood_kwargs(2, 3)["step_mri"] == 3
    assert patient.read_tumor_ic(tmp_path / "TumorIC.txt") == (0.28, 0.67, 0.35)
    (tmp_path / "InputParameters.txt").write_text("0.13\n0.025\n150\n")
    assert patient.read_input_parameters(tmp_path / "InputParameters.txt") == (0.13, 0.025, 150.0)
    (tmp_path / "short.txt").write_text("0.13 0.025\n")
    with pytest.raises(ValueError):
        patient.read_input_parameters(tmp_path / "short.txt")
    obs2 = patient.load_observations(tmp_path, pet=False)
    assert obs2.pet is None and obs2.roi is None
    with pytest.raises(GbfkError):
        patient.load_observations(tmp_path / "nothing")
