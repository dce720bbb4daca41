"""The C ABI library loads and exports every symbol include/gbfk.h declares
(no compute: this runs without a GPU)."""
import ctypes
import re
from pathlib import Path

from gliomasolver_b200 import _lib
from gliomasolver_b200.build import build_library

ROOT = Path(__file__).resolve().parents[1]


def header_symbols():
    text = (ROOT / "include" / "gbfk.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gbfk_[a-z_]+)\s*\(", text)))


def test_header_declares_the_binding():
    assert header_symbols() == sorted(_lib.EXPORTS)


def test_library_exports_every_declared_symbol():
    path = build_library()
    L = ctypes.CDLL(str(path))
    for name in header_symbols():
        assert hasattr(L, name), name


def test_create_rejects_bad_config_without_touching_the_device():
    L = _lib.load(build_library())
    h = ctypes.c_void_p()
    bad = _lib.Config(7, 16, 0, None)          # unknown precision
    assert L.gbfk_create(ctypes.byref(bad), ctypes.byref(h)) == 1
    bad = _lib.Config(_lib.GBFK_F32, 0, 0, None)  # empty pool
    assert L.gbfk_create(ctypes.byref(bad), ctypes.byref(h)) == 1
    assert not h.value
    assert L.gbfk_destroy(None) == 0
    assert L.gbfk_rd_step(None, 0.0, 0.0, 0.0, 0.0, 1, 0) == 1


def test_product_does_not_import_the_oracle():
    pkg = ROOT / "gliomasolver_b200"
    for p in pkg.rglob("*.py"):
        src = p.read_text()
        assert "oracle" not in re.findall(r"^\s*(?:from|import)\s+(\w+)", src, flags=re.M), p
    for p in list(pkg.rglob("*.cu")) + list(pkg.rglob("*.cuh")):
        assert "rd_oracle" not in p.read_text(), p
