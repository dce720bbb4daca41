"""Seeded synthetic brain anatomy and tumour initial condition.

The reference maps patient GM/WM/CSF volumes onto the grid in
``Glioma_ReactionDiffusion::_ic`` (Glioma/Glioma_ReactionDiffusion.cpp:79-172):
CSF wins a majority vote against tissue (``:144-147``), after which ``p_w`` and
``p_g`` are the normalised white/grey-matter fractions (``:149-151``).  No
patient data ships with the reference, so this module builds a synthetic
anatomy of the same kind from a seed:

* a brain ellipsoid centred in the unit cube with semi-axes
  ``(0.40, 0.34, 0.30) * scale``;
* an inner white-matter ellipsoid (semi-axes 0.62 of the brain's) whose radius
  is perturbed by a seeded, smooth (low-order trigonometric) noise field;
  ``P_WM`` falls off with a ``tanh`` edge;
* ``P_GM = 1 - P_WM`` inside the brain;
* two CSF ventricle ellipsoids with ``P_CSF = 1``.  By the reference's
  majority vote these cells get ``p_w = p_g = 0``.

The tumour initial condition is ``c0 = exp(-|x - x0|^2 / (2 (2h)^2))`` with
``x0`` a seeded uniformly chosen white-matter voxel (``P_WM > 0.5``), and
``c0 = 0`` where there is no tissue, as in the reference's IC
(``Glioma_ReactionDiffusion.cpp:155-164`` only places tumour where
``pGM + pWM > 0``).

Cell positions are vertex-centred, ``x_i = i / n`` (MRAG's
``BlockInfo::pos``, MRAG/MRAGcore/MRAGCommon.h:199, with the
Interp2ndOrder wavelets' zero centring offset).  Arrays are float64 and
indexed ``[z, y, x]`` (x fastest in memory), the block layout of
MRAG/MRAGcore/MRAGBlock.h:40.
"""
from __future__ import annotations

import numpy as np

BRAIN_SEMI_AXES = (0.40, 0.34, 0.30)
WM_FRACTION = 0.62
WM_EDGE = 0.06
VENTRICLES = (
    # centre offset from the brain centre (fraction of semi-axes), semi-axes (fraction of brain)
    ((-0.22, 0.05, 0.05), (0.12, 0.28, 0.14)),
    ((+0.22, 0.05, 0.05), (0.12, 0.28, 0.14)),
)
N_NOISE_MODES = 6


def _noise_field(rng: np.random.Generator, ux, uy, uz):
    """Smooth seeded perturbation of the white-matter radius on the unit sphere."""
    out = np.zeros_like(ux)
    for _ in range(N_NOISE_MODES):
        k = rng.integers(1, 4, size=3).astype(np.float64)
        phase = rng.uniform(0.0, 2.0 * np.pi)
        amp = rng.uniform(0.02, 0.06)
        out += amp * np.sin(k[0] * ux + k[1] * uy + k[2] * uz + phase)
    return out


def make_anatomy(n: int, seed: int = 0, scale: float = 1.0):
    """Return ``(p_w, p_g, p_csf)`` on an ``n^3`` vertex-centred grid.

    ``p_w`` and ``p_g`` already went through the reference's majority vote and
    normalisation, so they can be written straight into the blocks.
    """
    rng = np.random.default_rng(seed)
    x = np.arange(n, dtype=np.float64) / n
    zz, yy, xx = np.meshgrid(x, x, x, indexing="ij")
    a = np.array(BRAIN_SEMI_AXES) * scale
    dx, dy, dz = xx - 0.5, yy - 0.5, zz - 0.5
    rb = np.sqrt((dx / a[0]) ** 2 + (dy / a[1]) ** 2 + (dz / a[2]) ** 2)
    brain = rb <= 1.0

    aw = a * WM_FRACTION
    rw = np.sqrt((dx / aw[0]) ** 2 + (dy / aw[1]) ** 2 + (dz / aw[2]) ** 2)
    inv = 1.0 / np.maximum(rw, 1e-12)
    noise = _noise_field(rng, dx / aw[0] * inv, dy / aw[1] * inv, dz / aw[2] * inv)
    wm_raw = 0.5 * (1.0 - np.tanh((rw - (1.0 + noise)) / (WM_EDGE / WM_FRACTION)))
    p_wm = np.where(brain, wm_raw, 0.0)
    p_gm = np.where(brain, 1.0 - p_wm, 0.0)

    p_csf = np.zeros_like(p_wm)
    for off, semi in VENTRICLES:
        c = 0.5 + np.array(off) * a
        s = np.array(semi) * a
        rv = ((xx - c[0]) / s[0]) ** 2 + ((yy - c[1]) / s[1]) ** 2 + ((zz - c[2]) / s[2]) ** 2
        p_csf = np.where(rv <= 1.0, 1.0, p_csf)

    # majority vote and normalisation as in Glioma_ReactionDiffusion.cpp:144-151
    tissue = p_wm + p_gm
    csf_wins = p_csf > tissue
    p_csf = np.where(csf_wins, 1.0, 0.0)
    p_wm = np.where(csf_wins, 0.0, p_wm)
    p_gm = np.where(csf_wins, 0.0, p_gm)
    tissue = p_wm + p_gm
    safe = np.where(tissue > 0.0, tissue, 1.0)
    p_w = np.where(tissue > 0.0, p_wm / safe, 0.0)
    p_g = np.where(tissue > 0.0, p_gm / safe, 0.0)
    return np.ascontiguousarray(p_w), np.ascontiguousarray(p_g), np.ascontiguousarray(p_csf)


def pick_origin(p_w: np.ndarray, seed: int = 0, count: int = 1):
    """Seeded uniform choice of white-matter voxels (``P_WM > 0.5``); returns
    ``count`` positions ``(x, y, z)`` in unit-cube coordinates."""
    n = p_w.shape[0]
    rng = np.random.default_rng(seed + 7919)
    cand = np.flatnonzero(p_w.ravel() > 0.5)
    idx = cand[rng.integers(0, cand.size, size=count)]
    iz, iy, ix = np.unravel_index(idx, p_w.shape)
    return np.stack([ix / n, iy / n, iz / n], axis=1)


def tumor_ic(n: int, x0, p_w: np.ndarray, p_g: np.ndarray):
    """``c0 = exp(-|x - x0|^2 / (2 (2h)^2))`` where there is tissue, else 0."""
    h = 1.0 / n
    x = np.arange(n, dtype=np.float64) / n
    gx = np.exp(-((x - x0[0]) ** 2) / (2.0 * (2.0 * h) ** 2))
    gy = np.exp(-((x - x0[1]) ** 2) / (2.0 * (2.0 * h) ** 2))
    gz = np.exp(-((x - x0[2]) ** 2) / (2.0 * (2.0 * h) ** 2))
    c0 = gz[:, None, None] * gy[None, :, None] * gx[None, None, :]
    return np.ascontiguousarray(np.where(p_w + p_g > 0.0, c0, 0.0))


def make_case(n: int, seed: int = 0, scale: float = 1.0):
    """Anatomy plus initial condition: ``(p_w, p_g, c0, x0)``."""
    p_w, p_g, _ = make_anatomy(n, seed, scale)
    x0 = pick_origin(p_w, seed)[0]
    c0 = tumor_ic(n, x0, p_w, p_g)
    return p_w, p_g, c0, x0
