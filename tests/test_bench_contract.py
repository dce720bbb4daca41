"""The reference arm of bench.py (`--impl reference`) on the CPU, alone and
under torchrun with two ranks: one JSON line with the metric, unit and config
of the GPU arm, `impl`, a `cpu_baseline` that describes the run and an `e2e`
without copies."""
import json
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def test_reference_arm_prints_one_json_line():
    if not (ROOT / "oracle" / "_ref" / "ref_harness_f32").exists():
        pytest.skip("oracle/_ref is built only where the reference sources are")
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "3"],
                       cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "RD cell-updates/s & % HBM roofline" and d["unit"] == "cell-updates/s"
    assert d["value"] > 0 and d["higher_is_better"] is True and d["steps"] == 1 and d["warmup"] >= 3
    assert d["config"]["n"] == 256 and d["config"]["precision"] == "f32"
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == d["value"] and cb["cores"] >= 1 and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_under_torchrun_prints_on_rank_0_only():
    """Launched like the driver's N>1 runs (torchrun, two ranks on 127.0.0.1):
    rank 0 alone runs and prints the line; the other rank exits 0 without
    work."""
    if not (ROOT / "oracle" / "_ref" / "ref_harness_f32").exists():
        pytest.skip("oracle/_ref is built only where the reference sources are")
    import socket

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    r = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
                        "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "3"],
                       cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
