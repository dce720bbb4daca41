"""Config 2's adaptive schedule on the reference's own MRAG grid.

oracle/_ref/adaptive_run_{f64,f32} (built from the reference sources and
include/gbfk_mrag.hpp, see oracle/adaptive_run.cpp) refines a level-2 grid up
to level 5 (256^3-equivalent) with the reference's AutomaticRefinement
(refine tolerance 1e-3), compresses it once (tolerance 1e-4), then steps the
RD equation (Dw = 0.2 cm^2/day, rho = 0.05/day) re-adapting every 20 steps:
either with the reference's own step ("ref", the oracle) or with the leaves
resident on the GPU between adaptations ("gpu": one gbfk_rd_step call per
20 steps).  The block lists after every adaptation must be identical and
the final fields bit-identical; the FP32-storage run is compared with the
FP64 oracle (relative L2 on the finest uniform grid)."""
import json
import os
import subprocess

import numpy as np
import pytest

from gliomasolver_b200.anatomy import make_case

pytestmark = pytest.mark.gpu
REF = __import__("pathlib").Path(__file__).resolve().parents[1] / "oracle" / "_ref"
MAXLEVEL, RTOL, CTOL, EVERY = 5, "1e-3", "1e-4", 20


@pytest.fixture(scope="module")
def dense_input(tmp_path_factory):
    n = 8 << MAXLEVEL
    pw, pg, c0, _ = make_case(n, 0)
    path = tmp_path_factory.mktemp("adaptive") / "in.bin"
    with open(path, "wb") as f:
        f.write(np.int32(n).tobytes())
        for a in (pw, pg, c0):
            f.write(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    return path


def _run(prec, mode, inp, steps, out_dir):
    exe = REF / f"adaptive_run_{prec}"
    if not exe.exists():
        pytest.skip("oracle/_ref/adaptive_run is built only where the reference sources are")
    out = out_dir / f"{prec}_{mode}_{steps}.bin"
    r = subprocess.run([str(exe), str(inp), str(MAXLEVEL), RTOL, CTOL, str(steps), str(EVERY), mode, str(out)],
                       capture_output=True, text=True, timeout=1200,
                       env=dict(os.environ, GBFK_ORACLE_THREADS=str(os.cpu_count() or 1)))
    assert r.returncode == 0, r.stderr[-2000:]
    rec = json.loads(r.stdout.strip().splitlines()[-1])
    with open(out, "rb") as f:
        n = int(np.frombuffer(f.read(4), dtype=np.int32)[0])
        phi = np.frombuffer(f.read(), dtype=np.float64).reshape(n, n, n)
    return rec, phi


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_block_lists_and_fields_match_the_reference(gbfk_lib, dense_input, tmp_path, prec):
    ref, a = _run(prec, "ref", dense_input, 100, tmp_path)
    gpu, b = _run(prec, "gpu", dense_input, 100, tmp_path)
    assert len(set(ref["blocks"])) > 1, ref          # the grid did re-adapt
    assert gpu["blocks"] == ref["blocks"] and gpu["hashes"] == ref["hashes"]
    assert np.array_equal(a, b)


def test_fp32_storage_against_the_fp64_oracle(gbfk_lib, dense_input, tmp_path):
    """FP32 storage on the GPU vs the reference's FP64 run, same schedule:
    the block lists agree and the relative L2 error of phi stays below 1e-5."""
    ref, a = _run("f64", "ref", dense_input, 2000, tmp_path)
    gpu, b = _run("f32", "gpu", dense_input, 2000, tmp_path)
    gpu64, c = _run("f64", "gpu", dense_input, 2000, tmp_path)
    rel = np.linalg.norm(b - a) / np.linalg.norm(a)
    print(json.dumps({"fp32_vs_fp64_rel_l2": rel, "blocks": ref["blocks"], "lists_match": gpu["hashes"] == ref["hashes"],
                      "ref_f64_step_s": ref["step_seconds"], "gpu_f32_step_s": gpu["step_seconds"],
                      "gpu_f64_step_s": gpu64["step_seconds"], "cell_updates": ref["cell_updates"]}))
    assert gpu64["hashes"] == ref["hashes"] and np.array_equal(c, a)
    assert gpu["hashes"] == ref["hashes"]
    assert rel <= 1e-5
