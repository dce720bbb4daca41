"""Generate the golden fixtures of the grid-adaptation functions from the
reference itself.

Runs the reference's own BlockFWT, Grid::refine (BlockSplitter) and
Grid::compress (BlockCollapser) on an adapted grid
(oracle/_ref/topo_harness_{f64,f32}, built by ``make -C oracle ref`` from
the reference sources; see oracle/topo_harness.cpp) and stores, per
precision: the ghost lists of the grid before the split (row lengths and
source deltas, for size), p_w, p_g and phi of its leaves, their spacings, the
reference's per-block wavelet details, a SHA-256 of the exact bytes of its
ReactionDiffusionOperator sweep (dphidt in Real) with the coefficients and a
strided subsample, the first eight split parents with their children's phi
and those of them that collapsed back with the parent's phi.

    python tests/golden/make_golden_topology.py      # needs oracle/_ref
"""
from __future__ import annotations

import hashlib
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle as O  # noqa: E402

OUT = Path(__file__).resolve().parent
# base grid 2^3 blocks, refined up to level 3 (tolerance 3e-2), every 12th leaf split
CASE = dict(base_bpd=2, maxlevel=4, refine_tol=3e-2, every=12)
KEEP = 8


def main():
    for prec in ("f64", "f32"):
        if not O.ref_topology_available(prec):
            raise SystemExit(f"oracle/_ref/topo_harness_{prec} is not built (make -C oracle ref)")
        d = O.ref_topology(precision=prec, **CASE)
        real = np.float64 if prec == "f64" else np.float32
        parents = d["split_parent"][:KEEP]
        kids = d["split_phi"].reshape(-1, 8, 512)[:KEEP]
        sel = d["collapse_parent"] < KEEP
        np.savez_compressed(
            OUT / f"topology_adapt_{prec}.npz",
            case=np.array([CASE["base_bpd"], CASE["maxlevel"], CASE["every"]]),
            refine_tol=np.float64(CASE["refine_tol"]),
            level=d["level"].astype(np.int8),
            row_len=np.diff(d["row_ptr"]).astype(np.uint8),
            src_delta=np.diff(d["src"], prepend=0).astype(np.int32),
            w0=d["w0"], w1=d["w1"], w2=d["w2"],
            p_w=d["p_w"], p_g=d["p_g"], phi=d["phi"], h=d["h"], detail=d["detail"],
            coeffs=d["coeffs"],
            rhs_sha256=np.frombuffer(hashlib.sha256(d["rhs"].astype(real).tobytes()).digest(), np.uint8),
            rhs_sample=d["rhs"][::997],
            split_parent=parents, split_phi=kids.ravel(),
            collapse_parent=d["collapse_parent"][sel],
            collapse_phi=d["collapse_phi"].reshape(-1, 512)[sel].ravel())
        print(prec, d["summary"])


if __name__ == "__main__":
    main()
