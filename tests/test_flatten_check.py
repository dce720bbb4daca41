"""The MRAG adapter's host side (include/gbfk_mrag.hpp) on the reference's own
adaptive grid: the ghost-list flattening, parallel over blocks, against a
plain serial restatement of the layout, at one and several threads, into
reused and fresh lists; the Cell gathers and scatters
(oracle/flatten_check.cpp, built with the reference's sources).  CPU only."""
import json
import os
import subprocess
from pathlib import Path

import pytest

EXE = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "flatten_check"


@pytest.mark.parametrize("maxlevel,rtol,ctol,threads", [(4, "1e-3", "1e-4", 1), (4, "1e-3", "1e-4", 4),
                                                        (4, "3e-4", "0", 7), (3, "0", "0", 3)])
def test_flatten_matches_the_serial_layout(maxlevel, rtol, ctol, threads):
    if not EXE.exists():
        pytest.skip("oracle/_ref/flatten_check is built only where the reference sources are")
    r = subprocess.run([str(EXE), str(maxlevel), rtol, ctol, str(threads)], capture_output=True, text=True,
                       timeout=300, env=dict(os.environ, GBFK_TBB_THREADS="2"))
    rec = json.loads(r.stdout.strip().splitlines()[-1])
    print(json.dumps(rec))
    assert r.returncode == 0 and rec["ok"], rec
    assert rec["leaves"] > 64 and rec["entries"] > 0
