"""Build libgbfk.so in-tree for sm_100a with nvcc (no JIT cache, no torch
extension machinery): the shared object sits next to this file and travels
with the source tree."""
from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
SOURCES = ["csrc/gbfk_kernels.cu", "csrc/gbfk_api.cu", "csrc/gbfk_static.cu", "csrc/gbfk_uq.cu", "csrc/gbfk_batch.cu",
           "csrc/gbfk_step_tma.cu", "csrc/gbfk_patient.cpp"]
OUT = HERE / "libgbfk.so"

NVCC_FLAGS = [
    "-O3", "-std=c++17",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    # the RD arithmetic must round exactly like the reference's CPU code
    "-fmad=false",
    "-Xcompiler", "-fPIC,-ffp-contract=off", "-shared",
]


def nvcc() -> str:
    cand = [os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"]
    for c in cand:
        if c and Path(c).exists():
            return c
    raise RuntimeError("nvcc not found")


def needs_build() -> bool:
    if not OUT.exists():
        return True
    mt = OUT.stat().st_mtime
    deps = [HERE / s for s in SOURCES] + list((HERE / "csrc").glob("*.cuh")) + [ROOT / "include" / "gbfk.h"]
    return any(d.stat().st_mtime > mt for d in deps if d.exists())


def build_library(force: bool = False, verbose: bool = False) -> Path:
    if not force and not needs_build():
        return OUT
    # a temporary name per process: ranks that build at the same time each
    # replace the library atomically with a complete file
    tmp = f"{OUT}.tmp{os.getpid()}"
    cmd = [nvcc(), *NVCC_FLAGS, "-I", str(ROOT / "include"), *[str(HERE / s) for s in SOURCES], "-o", tmp]
    if verbose:
        print(" ".join(cmd))
    try:
        subprocess.run(cmd, check=True)
        os.replace(tmp, OUT)
    finally:
        if os.path.exists(tmp):
            os.remove(tmp)
    return OUT


if __name__ == "__main__":
    print(build_library(force=True, verbose=True))
