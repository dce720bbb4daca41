"""The heat equation with a known solution on adaptive grids: the reference's
STDTestL3_Diffusion (MRAG/MRAGcore/MRAG_STDTestL3_Diffusion.h:108-170, a 2-D
diffusion run on a refined grid against exp(-8 pi^2 t) sin sin) restated for
this 3-D solver.  Parity with the reference pins the arithmetic; this pins
that coarse-fine ghost interpolation converges when the grid has several
levels.

dropin/_build/glioma_adaptive_f64 runs the RD step with rho = 0 and p_w = 1
everywhere (D = Dw in every cell, no no-flux switch): a Gaussian bump
    c(x, t) = 0.25 + 0.5 (sigma^2 / s^2)^(3/2) exp(-|x - x0|^2 / (2 s^2)),
    s^2 = sigma^2 + 2 D t,
on the periodic unit cube (its images are below 1e-40).  The reference's
AutomaticRefinement / AutomaticCompression (refine tolerance rtol, compress
rtol / 10; rtol = 0 refines every block to the finest level) lay out the grid
from the initial field and keep it for the whole run (every = 0).  Each leaf
cell's value sits at its vertex origin + h * index, the reference's
BlockInfo::pos (MRAGCommon.h:199-204), where the initial field is sampled
too.  Levels 3, 4 and 5 (64^3- to 256^3-equivalent) run the same physical
time (dt scales with h^2 exactly: 4x the steps per level).  Measured on a
B200 (relative L2 error at the leaves, against the bump's height):

    uniform (rtol 0)   L3 1.37e-4   L4 3.40e-5   L5 8.48e-6   (4.0x per level)
    rtol 1e-3 .. 1e-5 at L5: 1.96e-4, 7.20e-5, 2.33e-5 with 1324, 2899, 4285 of
    32768 blocks; rtol 1e-3 at L3, 1e-4 at L4, 1e-5 at L5: 1.77e-4, 5.78e-5,
    2.33e-5.
"""
import json
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
EXE = ROOT / "dropin" / "_build" / "glioma_adaptive_f64"
SIGMA, X0, DW_DAY, L_CM = 0.06, (0.5, 0.47, 0.53), 0.2, 25.6
STEPS = {3: 45, 4: 180, 5: 720}


def _exact(x, y, z, t_day):
    D = DW_DAY / (L_CM * L_CM)
    s2 = SIGMA ** 2 + 2.0 * D * t_day
    r2 = (x - X0[0]) ** 2 + (y - X0[1]) ** 2 + (z - X0[2]) ** 2
    return 0.25 + 0.5 * (SIGMA ** 2 / s2) ** 1.5 * np.exp(-r2 / (2.0 * s2))


_RUNS = {}


def _run(level, rtol, tmp):
    key = (level, rtol)
    if key in _RUNS:
        return _RUNS[key]
    if not EXE.exists():
        pytest.skip("dropin/_build is built only where the reference sources are")
    n = 8 << level
    i = np.arange(n) / n  # vertex positions
    z, y, x = np.meshgrid(i, i, i, indexing="ij")
    inp, out = tmp / "heat.bin", tmp / "heat.out"
    with open(inp, "wb") as f:
        f.write(np.int32(n).tobytes())
        f.write(np.ones(n ** 3).tobytes())       # p_w
        f.write(np.zeros(n ** 3).tobytes())      # p_g
        f.write(np.ascontiguousarray(_exact(x, y, z, 0.0)).tobytes())
    r = subprocess.run([str(EXE), str(inp), str(level), repr(rtol), repr(rtol / 10), str(STEPS[level]), "0", str(out),
                        str(DW_DAY), "0"], capture_output=True, text=True, timeout=900,
                       env=dict(os.environ, GBFK_TBB_THREADS=str(os.cpu_count() or 1)))
    assert r.returncode == 0, r.stderr[-2000:]
    info = json.loads(r.stdout.strip().splitlines()[-1])
    with open(out, "rb") as f:
        assert int(np.frombuffer(f.read(4), dtype=np.int32)[0]) == n
        u = np.frombuffer(f.read(), dtype=np.float64).reshape(n, n, n)
    lev = np.fromfile(str(out) + ".levels", dtype=np.int8).reshape(n, n, n)
    t_day = STEPS[level] * info["dt"]
    # one sample per leaf cell, at its vertex: finest cells whose coordinates
    # are multiples of r = 2^(level - leaf level), weighted by r^3
    r_map = 1 << (level - lev.astype(np.int64))
    idx = np.arange(n)
    first = ((idx[None, None, :] % r_map) == 0) & ((idx[None, :, None] % r_map) == 0) & \
            ((idx[:, None, None] % r_map) == 0)
    err = (u - _exact(x, y, z, t_day))[first]
    w = (r_map[first].astype(np.float64) / n) ** 3
    bump = 0.5 * (SIGMA ** 2 / (SIGMA ** 2 + 2.0 * DW_DAY / L_CM ** 2 * t_day)) ** 1.5
    res = {"level": level, "rtol": rtol, "t_day": t_day, "blocks": info["blocks"][0],
           "leaf_cells_per_level": {int(k): int(np.count_nonzero(lev[first] == k)) for k in np.unique(lev)},
           "rel_l2": float(np.sqrt(np.sum(w * err ** 2)) / bump), "rel_max": float(np.abs(err).max() / bump)}
    _RUNS[key] = res
    return res


def test_uniform_grids_converge_at_second_order(gbfk_lib, tmp_path):
    """rtol = 0: every block at the finest level; the error falls 4x per level
    (second order in h, dt ~ h^2), the physical time being the same."""
    runs = [_run(level, 0.0, tmp_path) for level in (3, 4, 5)]
    print(json.dumps(runs))
    for a, b in zip(runs, runs[1:]):
        assert b["t_day"] == pytest.approx(a["t_day"], rel=1e-12)
        assert len(b["leaf_cells_per_level"]) == 1
        assert 3.5 < a["rel_l2"] / b["rel_l2"] < 4.5
    assert runs[-1]["rel_l2"] < 1e-5


def test_adaptive_grids_approach_the_uniform_error(gbfk_lib, tmp_path):
    """Multi-level grids (the reference's refinement of the bump, coarse
    blocks elsewhere): at the finest level 5 the error falls with the
    tolerance towards the uniform grid's, and refining the tolerance with
    the level (1e-3 at level 3, 1e-4 at 4, 1e-5 at 5) converges too."""
    uni = _run(5, 0.0, tmp_path)
    at5 = [_run(5, rtol, tmp_path) for rtol in (1e-3, 1e-4, 1e-5)]
    seq = [_run(3, 1e-3, tmp_path), _run(4, 1e-4, tmp_path), at5[2]]
    print(json.dumps({"uniform_l5": uni, "l5": at5, "sequence": seq}))
    for r in at5:
        assert len(r["leaf_cells_per_level"]) >= 3 and r["blocks"] < uni["blocks"] // 4
    assert at5[0]["rel_l2"] > 2 * at5[1]["rel_l2"] > 4 * at5[2]["rel_l2"]
    assert uni["rel_l2"] < at5[2]["rel_l2"] < 4 * uni["rel_l2"]
    for a, b in zip(seq, seq[1:]):
        assert a["rel_l2"] > 2 * b["rel_l2"]
