"""Generate the golden fixture of the anatomy mapping from the reference itself.

Runs the reference's own Glioma_ReactionDiffusion::_ic
(oracle/_ref/ic_harness_{f64,f32}, built by ``make -C oracle ref`` from the
reference sources) on small seeded GM/WM/CSF volumes written as Matrix
files, and stores the volumes, the tumour centres and the reference's cells
(p_w, p_g, p_csf, phi and L) for each grid and precision.

    python tests/golden/make_golden_anatomy.py          # needs oracle/_ref
"""
from __future__ import annotations

import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle as O  # noqa: E402

OUT = Path(__file__).resolve().parent / "anatomy_ic.npz"
SHAPE = (12, 14, 13)            # [z, y, x]: the longest side (y) sets the voxel spacing
# (blocks per direction, tumour centre): centres next to a grid vertex so that
# cells fall in the smoothing band of the ball
GRIDS = ((2, (0.5 + 0.006, 0.5 - 0.004, 0.5 + 0.003)), (3, (0.25 + 0.004, 0.375 + 0.002, 0.3125 - 0.005)))


def volumes(seed: int = 11):
    """Random fractions with the cases the mapping branches on: CSF ties with
    the tissue sum, unnormalised fractions (CSF above a tissue sum >= 1),
    tissue below the tumour's 0.001 threshold, and empty voxels."""
    rng = np.random.default_rng(seed)
    gm = np.round(rng.uniform(0, 1, SHAPE) * 64) / 64
    wm = np.round(rng.uniform(0, 1, SHAPE) * 64) / 64
    csf = np.round(rng.uniform(0, 1, SHAPE) ** 3 * 64) / 64
    m = rng.uniform(0, 1, SHAPE)
    tie = m < 0.08
    csf[tie] = (gm + wm)[tie]
    big = m > 0.92
    gm[big] *= 1.5
    wm[big] *= 1.5
    csf[big] = 2.75
    tiny = (m > 0.30) & (m < 0.36)
    gm[tiny], wm[tiny], csf[tiny] = 2e-4, 3e-4, 0.0
    empty = (m > 0.40) & (m < 0.44)
    gm[empty] = wm[empty] = csf[empty] = 0.0
    # the voxels under the tumour centres: tiny tissue, so the ball's tissue tests matter
    for bpd, tic in GRIDS:
        v = [int(np.floor(t * max(SHAPE))) for t in tic]
        gm[v[2], v[1], v[0]], wm[v[2], v[1], v[0]], csf[v[2], v[1], v[0]] = 4e-4, 5e-4, 0.0
    return gm, wm, csf


def main():
    if not O.ref_ic_available("f64") or not O.ref_ic_available("f32"):
        sys.exit("oracle/_ref/ic_harness is not built: run `make -C oracle ref` where the reference sources are")
    gm, wm, csf = volumes()
    out = {"gm": gm, "wm": wm, "csf": csf}
    with tempfile.TemporaryDirectory() as td:
        prefix = str(Path(td) / "P_")
        for k, v in (("GM", gm), ("WM", wm), ("CSF", csf)):
            O.write_matrix3d(prefix + k + ".dat", v)
        for bpd, tic in GRIDS:
            out[f"tic_bpd{bpd}"] = np.array(tic)
            for prec in ("f64", "f32"):
                r = O.ref_map_anatomy(prefix, bpd, tic, prec)
                R = np.float64 if prec == "f64" else np.float32
                for k in ("p_w", "p_g", "p_csf", "phi"):
                    assert np.array_equal(r[k].astype(R).astype(np.float64), r[k])
                    out[f"{prec}_bpd{bpd}_{k}"] = r[k].astype(R)
                out[f"{prec}_bpd{bpd}_L"] = np.array(r["L"])
                band = int(np.count_nonzero((r["phi"] > 0) & (r["phi"] < 1)))
                print(f"bpd {bpd} {prec}: L {r['L']!r}, {band} cells in the smoothing band")
    np.savez_compressed(OUT, **out)
    print(OUT, OUT.stat().st_size, "bytes")


if __name__ == "__main__":
    main()
