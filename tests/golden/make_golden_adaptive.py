"""Generates tests/golden/adaptive_t300_f64.json: the block-list record of the
reference's own adaptive run over config 2's full horizon (T = 300 days).

Input: the seeded synthetic case make_case(256, 0) (p_w, p_g and the Gaussian
c0 on the 256^3 finest grid).  The run is oracle/_ref/adaptive_run_f64 (built
from the reference sources by oracle/Makefile): the reference's grid refined
from level 2 to level 5 and compressed once, then 36364 RD steps of
Dw = 0.2 cm^2/day, rho = 0.05/day at the reference's dt for the finest
spacing (make_schedule(0.2, 0.05, 300, 25.6, 32, "f64")), re-adapting every
20 steps (one refinement loop at tolerance 1e-3, compression to convergence at
1e-4), every step and adaptation by the reference's own code.  The record
keeps the number of leaves and the FNV-1a hash of the sorted leaf list after
every adaptation, dt, the timings and the SHA-256 of the final phi sampled on
the finest grid (float64, x fastest).  About half an hour on 8 host cores.

    python tests/golden/make_golden_adaptive.py [threads]
"""
import hashlib
import json
import os
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from gliomasolver_b200.anatomy import make_case  # noqa: E402
from gliomasolver_b200.schedule import make_schedule  # noqa: E402


def main():
    threads = sys.argv[1] if len(sys.argv) > 1 else str(os.cpu_count() or 1)
    n, maxlevel, every = 256, 5, 20
    steps = make_schedule(0.2, 0.05, 300.0, 25.6, n // 8, "f64").nsteps
    pw, pg, c0, _ = make_case(n, 0)
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        with open(fin, "wb") as f:
            f.write(np.int32(n).tobytes())
            for a in (pw, pg, c0):
                f.write(np.ascontiguousarray(a, dtype=np.float64).tobytes())
        r = subprocess.run([str(ROOT / "oracle" / "_ref" / "adaptive_run_f64"), fin, str(maxlevel), "1e-3", "1e-4",
                            str(steps), str(every), "ref", fout], check=True, capture_output=True, text=True,
                           env=dict(os.environ, GBFK_TBB_THREADS=threads))
        rec = json.loads(r.stdout.strip().splitlines()[-1])
        with open(fout, "rb") as f:
            f.read(4)
            rec["phi_sha256"] = hashlib.sha256(f.read()).hexdigest()
    rec["input"] = "make_case(256, 0): p_w, p_g, c0 as float64 on the finest grid"
    rec["host_threads"] = int(threads)
    (ROOT / "tests" / "golden" / "adaptive_t300_f64.json").write_text(json.dumps(rec) + "\n")


if __name__ == "__main__":
    main()
