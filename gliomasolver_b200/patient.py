"""Patient data for the RD path: Matrix files, the anatomy mapping and the
likelihood inputs.

The reference reads every volume through its ``Matrix`` classes
(Glioma/Matrix.h; the likelihood program has its own copy of the same file
in tools/pi4u_lite/Inference/Likelihood/source/Matrix.h): an int32 magic
number 1234, int32 dim (2 or 3), the int32 sizes with x first, an int32 type
id (0 double, 1 float, 2 int32) and the values, x fastest.  It maps the
patient's GM/WM/CSF volumes and the tumour initial condition onto its grid
in ``Glioma_ReactionDiffusion::_ic`` (Glioma/Glioma_ReactionDiffusion.cpp:
79-172) and reads the observations of the likelihood from tumT1c.dat,
tumFLAIR.dat, tumPET.dat, ROI.dat and LikelihoodInput.txt
(tools/pi4u_lite/Inference/Likelihood/source/HGG_Likelihood.cpp:11-36,
40-128).

All file parsing and the mapping run in libgbfk (gbfk_matrix_*,
gbfk_map_anatomy); this module converts between those calls and numpy.
Volumes are numpy arrays indexed ``[z, y, x]`` (x fastest in memory, the
Matrix layout); 2-D matrices are ``[y, x]``.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import GbfkError

TID_DOUBLE, TID_FLOAT, TID_INT = 0, 1, 2


def _host_check(rc: int):
    if rc != _lib.GBFK_OK:
        raise GbfkError(rc, _lib.load().gbfk_host_last_error().decode(errors="replace"))


def _path(p) -> bytes:
    return os.fsencode(os.fspath(p))


@dataclass
class MatrixInfo:
    dim: int
    sizes: tuple   # (nx, ny[, nz])
    type_id: int


def matrix_info(path) -> MatrixInfo:
    """Header of a Matrix file (Matrix.h:71-88 and the type id of :141-169)."""
    L = _lib.load()
    dim, tid = ctypes.c_int(), ctypes.c_int()
    sizes = (ctypes.c_int * 3)()
    _host_check(L.gbfk_matrix_info(_path(path), ctypes.byref(dim), ctypes.byref(sizes), ctypes.byref(tid)))
    return MatrixInfo(dim.value, tuple(sizes[:dim.value]), tid.value)


def read_matrix(path) -> np.ndarray:
    """Values of a Matrix file as float64, as ``MatrixD2D``/``MatrixD3D<double>``
    load them (Matrix.h:116-169,437-445,656-665): shape ``(nz, ny, nx)`` for
    a 3-D file, ``(ny, nx)`` for a 2-D one."""
    info = matrix_info(path)
    out = np.empty(tuple(reversed(info.sizes)), dtype=np.float64)
    _host_check(_lib.load().gbfk_matrix_read(_path(path), out.ctypes.data_as(ctypes.c_void_p), out.size))
    return out


def write_matrix(path, values, type_id: int = TID_DOUBLE):
    """Write a 2-D ``[y, x]`` or 3-D ``[z, y, x]`` array as a Matrix file with
    the given type id (Matrix.h:184-240,390-411,609-631)."""
    a = np.ascontiguousarray(values, dtype=np.float64)
    if a.ndim not in (2, 3):
        raise ValueError("a Matrix file holds a 2-D or 3-D array")
    sizes = (ctypes.c_int * 3)(*(list(reversed(a.shape)) + [0] * (3 - a.ndim)))
    _host_check(_lib.load().gbfk_matrix_write(_path(path), a.ndim, ctypes.byref(sizes), int(type_id),
                                              a.ctypes.data_as(ctypes.c_void_p)))


@dataclass
class PatientAnatomy:
    """The reference's cells after ``_ic`` on the uniform grid of
    ``blocks_per_dim`` blocks per direction, dense ``n^3`` (n = 8 *
    blocks_per_dim, ``[z, y, x]``) in the grid's Real."""
    p_w: np.ndarray
    p_g: np.ndarray
    p_csf: np.ndarray
    phi: np.ndarray
    tissue: np.ndarray   # p_g + p_w after the CSF vote, before normalisation
    L_cm: float          # characteristic length: longest volume side * 0.1 cm
    blocks_per_dim: int
    precision: str


def map_anatomy(gm, wm, csf, blocks_per_dim: int, tumor_ic, precision: str = "f64") -> PatientAnatomy:
    """``Glioma_ReactionDiffusion::_ic`` (Glioma_ReactionDiffusion.cpp:79-172)
    on GM/WM/CSF volumes of equal shape ``[z, y, x]`` (gbfk_map_anatomy)."""
    vols = [np.ascontiguousarray(v, dtype=np.float64) for v in (gm, wm, csf)]
    if vols[0].ndim != 3 or any(v.shape != vols[0].shape for v in vols):
        raise ValueError("GM, WM and CSF must be 3-D volumes of one shape")
    if precision not in ("f64", "f32"):
        raise ValueError("precision is 'f64' or 'f32'")
    dtype = np.float64 if precision == "f64" else np.float32
    n = 8 * int(blocks_per_dim)
    outs = [np.empty((n, n, n), dtype=dtype) for _ in range(5)]
    msize = (ctypes.c_int * 3)(*reversed(vols[0].shape))
    tic = (ctypes.c_double * 3)(*[float(v) for v in tumor_ic])
    L = ctypes.c_double()
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    _host_check(_lib.load().gbfk_map_anatomy(
        _lib.GBFK_F64 if precision == "f64" else _lib.GBFK_F32, int(blocks_per_dim), ctypes.byref(msize),
        *(P(v) for v in vols), ctypes.byref(tic), *(P(o) for o in outs), ctypes.byref(L)))
    return PatientAnatomy(*outs, L.value, int(blocks_per_dim), precision)


def load_patient(prefix, blocks_per_dim: int, tumor_ic, precision: str = "f64") -> PatientAnatomy:
    """Read ``{prefix}GM.dat``, ``{prefix}WM.dat`` and ``{prefix}CSF.dat`` (the
    reference's -PatFileName prefix, Glioma_ReactionDiffusion.cpp:84-89) and
    map them with the tumour at ``tumor_ic``."""
    prefix = os.fspath(prefix)
    gm, wm, csf = (read_matrix(f"{prefix}{k}.dat") for k in ("GM", "WM", "CSF"))
    return map_anatomy(gm, wm, csf, blocks_per_dim, tumor_ic, precision)


def read_tumor_ic(path="TumorIC.txt") -> tuple:
    """The tumour centre of a UQ run: three numbers (Glioma_ReactionDiffusion.cpp:39-52)."""
    with open(path) as f:
        vals = f.read().split()
    if len(vals) < 3:
        raise ValueError(f"{path}: expected three numbers")
    return tuple(float(v) for v in vals[:3])


def read_input_parameters(path="InputParameters.txt") -> tuple:
    """Dw [cm^2/day], rho [1/day] and Tend [day] of a UQ forward run: three
    numbers (Glioma_ReactionDiffusion.cpp:280-293), for make_schedule."""
    with open(path) as f:
        vals = f.read().split()
    if len(vals) < 3:
        raise ValueError(f"{path}: expected three numbers")
    return tuple(float(v) for v in vals[:3])


@dataclass
class Observations:
    """Inputs of the likelihood step, ready for ``set_observations`` and
    ``log_likelihood`` of a BlockPool or a Batch."""
    t1c: np.ndarray
    flair: np.ndarray
    pet: np.ndarray | None
    roi: np.ndarray | None   # (npoints, 3) int32 voxel triples (x, y, z)
    params: dict             # pet_sigma2, pet_scale, t1_uc, t2_uc, slope

    def likelihood_kwargs(self, step_pet: int = 1, step_mri: int = 1) -> dict:
        return dict(self.params, step_pet=int(step_pet), step_mri=int(step_mri))


def read_likelihood_input(path="LikelihoodInput.txt") -> dict:
    """PETsigma2, PETscale, T1uc, T2uc, slope (HGG_Likelihood.cpp:13-27)."""
    with open(path) as f:
        vals = f.read().split()
    if len(vals) < 5:
        raise ValueError(f"{path}: expected five numbers")
    keys = ("pet_sigma2", "pet_scale", "t1_uc", "t2_uc", "slope")
    return {k: float(v) for k, v in zip(keys, vals[:5])}


def read_roi(path="ROI.dat") -> np.ndarray:
    """The -bROI voxel list: a 2-D Matrix with nx = points and ny = 3 whose
    element (i, j) is coordinate j of point i, truncated to int
    (HGG_Likelihood.cpp:105-115)."""
    m = read_matrix(path)
    if m.ndim != 2 or m.shape[0] != 3:
        raise ValueError(f"{path}: expected a 2-D Matrix of size (points, 3)")
    return np.ascontiguousarray(np.trunc(m.T).astype(np.int32))


def load_observations(directory=".", roi: bool = False, pet: bool = True) -> Observations:
    """The files the reference's likelihood program reads from its working
    directory: tumT1c.dat, tumFLAIR.dat, tumPET.dat (when ``pet``), ROI.dat
    (when ``roi``, the -bROI 1 flag) and LikelihoodInput.txt."""
    d = os.fspath(directory)
    t1c = read_matrix(os.path.join(d, "tumT1c.dat"))
    flair = read_matrix(os.path.join(d, "tumFLAIR.dat"))
    pet_v = read_matrix(os.path.join(d, "tumPET.dat")) if pet else None
    roi_v = read_roi(os.path.join(d, "ROI.dat")) if roi else None
    params = read_likelihood_input(os.path.join(d, "LikelihoodInput.txt"))
    return Observations(t1c, flair, pet_v, roi_v, params)
