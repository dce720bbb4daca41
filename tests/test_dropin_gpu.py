"""The drop-in on adaptive grids built by the reference's own MRAG code.

oracle/_ref/dropin_demo_{f64,f32} (built from the reference sources and
include/gbfk_mrag.hpp, see oracle/dropin_demo.cpp) refines a level-2 grid with
the reference's AutomaticRefinement, then compares, bit for bit: the wavelet
details, RD steps through the drop-in BlockProcessing policy and through one
resident gbfk_rd_step call, split and collapse.  The ghost lists are the
reference's own BoundaryInfo, coarse-fine faces included."""
import json
import os
import subprocess
import tempfile
from pathlib import Path

import numpy as np
import pytest

from gliomasolver_b200.anatomy import make_case

pytestmark = pytest.mark.gpu
REF = Path(__file__).resolve().parents[1] / "oracle" / "_ref"


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_dropin_on_reference_adaptive_grid(gbfk_lib, prec):
    exe = REF / f"dropin_demo_{prec}"
    if not exe.exists():
        pytest.skip("oracle/_ref/dropin_demo is built only where the reference sources are")
    n, maxlevel = 128, 4
    pw, pg, c0, _ = make_case(n, 0)
    with tempfile.TemporaryDirectory() as td:
        fin = os.path.join(td, "in.bin")
        with open(fin, "wb") as f:
            f.write(np.int32(n).tobytes())
            for a in (pw, pg, c0):
                f.write(np.ascontiguousarray(a, dtype=np.float64).tobytes())
        r = subprocess.run([str(exe), fin, str(maxlevel), "1e-3", "20"], capture_output=True, text=True,
                           timeout=600, env=dict(os.environ, GBFK_TBB_THREADS=str(os.cpu_count() or 1)))
    assert r.returncode == 0, r.stderr[-2000:]
    rec = json.loads(r.stdout.strip().splitlines()[-1])
    assert len(rec["levels"]) >= 2, rec
    assert rec["coarse_fine_faces"] > 0, rec
    assert rec["fwt_max"] > 0
    for k in ("fwt_mismatch", "step_mismatch_dropin", "step_mismatch_deferred", "step_mismatch_resident",
              "split_mismatch", "collapse_mismatch"):
        assert rec[k] == 0, (k, rec)
    # the policy keeps phi on the device between topology changes: one upload
    # of the leaf set for the whole loop
    assert rec["dropin_uploads"] == 1, rec
    print({k: rec[k] for k in ("blocks", "steps", "reference_step_seconds", "dropin_step_seconds",
                               "deferred_step_seconds")})
    assert rec["split_parents"] > 0 and rec["collapsed"] == 1, rec
