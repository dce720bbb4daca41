"""ctypes binding of libgbfk.so (the C ABI declared in include/gbfk.h).

The library is built in-tree (``gliomasolver_b200/libgbfk.so``) by
``gliomasolver_b200.build.build_library``.  There is no fallback: if the
shared object is missing or does not load, every entry point raises.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libgbfk.so"

GBFK_OK = 0
STATUS = {
    0: "GBFK_OK",
    1: "GBFK_E_INVALID",
    2: "GBFK_E_CUDA",
    3: "GBFK_E_OOM",
    4: "GBFK_E_NAN",
    5: "GBFK_E_TIMEOUT",
    6: "GBFK_E_STATE",
    7: "GBFK_E_TOO_LARGE",
    8: "GBFK_E_IO",
}
STATUS_CODES = {v: k for k, v in STATUS.items()}
GBFK_F64, GBFK_F32 = 0, 1
GBFK_PHI, GBFK_PW, GBFK_PG = 0, 1, 2
# step kernels (gbfk_set_step_kernel)
STEP_KERNELS = {"auto": 0, "block": 1, "pipelined": 2, "run": 3}

# Every symbol include/gbfk.h declares (checked by the CPU test suite).
EXPORTS = (
    "gbfk_create", "gbfk_destroy", "gbfk_last_error", "gbfk_sync", "gbfk_launch_count",
    "gbfk_set_uniform", "gbfk_set_topology", "gbfk_num_blocks",
    "gbfk_upload_field", "gbfk_download_field", "gbfk_upload_dense", "gbfk_download_dense",
    "gbfk_rd_step", "gbfk_set_step_kernel", "gbfk_step_kernel",
    "gbfk_rd_rhs", "gbfk_cfl", "gbfk_rd_step_host", "gbfk_join_copies", "gbfk_fwt_details", "gbfk_split", "gbfk_collapse",
    "gbfk_rd_step_static",
    "gbfk_set_observations", "gbfk_uq_dump", "gbfk_log_likelihood",
    "gbfk_batch_create", "gbfk_batch_destroy", "gbfk_batch_last_error", "gbfk_batch_launch_count",
    "gbfk_batch_set_anatomy", "gbfk_batch_set_samples", "gbfk_batch_run", "gbfk_batch_samples_per_cta",
    "gbfk_batch_tile_shape", "gbfk_batch_graph_count",
    "gbfk_batch_download", "gbfk_batch_set_observations", "gbfk_batch_log_likelihood",
    "gbfk_forward_adjoint",
    "gbfk_probe_bounded_wait",
    "gbfk_host_last_error", "gbfk_matrix_info", "gbfk_matrix_read", "gbfk_matrix_write", "gbfk_map_anatomy",
)


class GbfkError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{STATUS.get(code, code)}: {message}")
        self.code = code


class Config(ctypes.Structure):
    _fields_ = [
        ("precision", ctypes.c_int),
        ("max_blocks", ctypes.c_int),
        ("device", ctypes.c_int),
        ("stream", ctypes.c_void_p),
    ]


class BlockInfo(ctypes.Structure):
    _fields_ = [
        ("slot", ctypes.c_int),
        ("level", ctypes.c_int),
        ("index", ctypes.c_int * 3),
        ("h", ctypes.c_double),
    ]


class LikelihoodParams(ctypes.Structure):
    _fields_ = [
        ("pet_sigma2", ctypes.c_double),
        ("pet_scale", ctypes.c_double),
        ("t1_uc", ctypes.c_double),
        ("t2_uc", ctypes.c_double),
        ("slope", ctypes.c_double),
        ("step_pet", ctypes.c_int),
        ("step_mri", ctypes.c_int),
    ]


class Sample(ctypes.Structure):
    _fields_ = [
        ("Dw", ctypes.c_double),
        ("Dg", ctypes.c_double),
        ("rho", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("nsteps", ctypes.c_int),
        ("anatomy", ctypes.c_int),
        ("x0", ctypes.c_double * 3),
        ("sigma", ctypes.c_double),
        ("ic", ctypes.c_int),
    ]


# initial conditions of a batch sample (enum gbfk_ic)
IC_KINDS = {"gaussian": 0, "ball": 1}

# gbfk_adjoint_params.flags
ADJ_TERM_MAGNITUDES = 1


class AdjointParams(ctypes.Structure):
    _fields_ = [
        ("Dw", ctypes.c_double), ("Dg", ctypes.c_double), ("rho", ctypes.c_double), ("dt", ctypes.c_double),
        ("nsteps", ctypes.c_int), ("nsnapshots", ctypes.c_int),
        ("x0", ctypes.c_double * 3), ("sigma", ctypes.c_double),
        ("t1_uc", ctypes.c_double), ("t2_uc", ctypes.c_double), ("slope", ctypes.c_double),
        ("flags", ctypes.c_int),
    ]


class AdjointResult(ctypes.Structure):
    _fields_ = [
        ("loss", ctypes.c_double), ("dDw", ctypes.c_double), ("drho", ctypes.c_double),
        ("dx0", ctypes.c_double * 3), ("forward_steps", ctypes.c_int64), ("adjoint_steps", ctypes.c_int64),
        ("dDw_abs", ctypes.c_double), ("drho_abs", ctypes.c_double),
    ]


class GhostCSR(ctypes.Structure):
    _fields_ = [
        ("nrows", ctypes.c_int64),
        ("row_ptr", ctypes.c_void_p),
        ("src", ctypes.c_void_p),
        ("w0", ctypes.c_void_p),
        ("w1", ctypes.c_void_p),
        ("w2", ctypes.c_void_p),
    ]


_lib = None


def load(path: Path | str | None = None):
    """Load libgbfk.so (once) and declare its signatures."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise ImportError(
            f"{p} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
            "(the CUDA extension is required; there is no CPU fallback)")
    L = ctypes.CDLL(str(p))
    P, I, I64, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_double
    sig = {
        "gbfk_create": (I, [ctypes.POINTER(Config), ctypes.POINTER(P)]),
        "gbfk_destroy": (I, [P]),
        "gbfk_last_error": (ctypes.c_char_p, [P]),
        "gbfk_sync": (I, [P]),
        "gbfk_launch_count": (I64, [P]),
        "gbfk_set_uniform": (I, [P, I]),
        "gbfk_set_topology": (I, [P, P, I, ctypes.POINTER(GhostCSR)]),
        "gbfk_num_blocks": (I, [P]),
        "gbfk_upload_field": (I, [P, I, P, I64, I64]),
        "gbfk_download_field": (I, [P, I, P, I64, I64]),
        "gbfk_upload_dense": (I, [P, I, P, I]),
        "gbfk_download_dense": (I, [P, I, P, I]),
        "gbfk_rd_step": (I, [P, D, D, D, D, I, I]),
        "gbfk_set_step_kernel": (I, [P, I]),
        "gbfk_step_kernel": (I, [P]),
        "gbfk_rd_rhs": (I, [P, D, D, D, P]),
        "gbfk_cfl": (I, [P, D, D, P]),
        "gbfk_rd_step_host": (I, [P, P, P, D, D, D, D, I]),
        "gbfk_join_copies": (I, [P]),
        "gbfk_fwt_details": (I, [P, P]),
        "gbfk_split": (I, [P, I, P, P]),
        "gbfk_collapse": (I, [P, I, P, P]),
        "gbfk_rd_step_static": (I, [I, I, P, P, P, P, D, D, D, D, P, I]),
        "gbfk_set_observations": (I, [P, I, P, P, P, P, I]),
        "gbfk_uq_dump": (I, [P, I, P]),
        "gbfk_log_likelihood": (I, [P, ctypes.POINTER(LikelihoodParams), P]),
        "gbfk_batch_create": (I, [ctypes.POINTER(Config), I, I, I, ctypes.POINTER(P)]),
        "gbfk_batch_destroy": (I, [P]),
        "gbfk_batch_last_error": (ctypes.c_char_p, [P]),
        "gbfk_batch_launch_count": (I64, [P]),
        "gbfk_batch_set_anatomy": (I, [P, I, P, P]),
        "gbfk_batch_set_samples": (I, [P, I, ctypes.POINTER(Sample)]),
        "gbfk_batch_run": (I, [P, I]),
        "gbfk_batch_samples_per_cta": (I, [P]),
        "gbfk_batch_tile_shape": (I, [P, ctypes.POINTER(I * 3)]),
        "gbfk_batch_graph_count": (I, [P]),
        "gbfk_batch_download": (I, [P, I, P]),
        "gbfk_batch_set_observations": (I, [P, P, P, P, P, I]),
        "gbfk_batch_log_likelihood": (I, [P, ctypes.POINTER(LikelihoodParams), I, P]),
        "gbfk_forward_adjoint": (I, [P, ctypes.POINTER(AdjointParams), ctypes.POINTER(AdjointResult), P]),
        "gbfk_probe_bounded_wait": (I, [I, ctypes.POINTER(D)]),
        "gbfk_host_last_error": (ctypes.c_char_p, []),
        "gbfk_matrix_info": (I, [ctypes.c_char_p, ctypes.POINTER(I), ctypes.POINTER(I * 3), ctypes.POINTER(I)]),
        "gbfk_matrix_read": (I, [ctypes.c_char_p, P, I64]),
        "gbfk_matrix_write": (I, [ctypes.c_char_p, I, ctypes.POINTER(I * 3), I, P]),
        "gbfk_map_anatomy": (I, [I, I, ctypes.POINTER(I * 3), P, P, P, ctypes.POINTER(D * 3), P, P, P, P, P,
                                 ctypes.POINTER(D)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L
