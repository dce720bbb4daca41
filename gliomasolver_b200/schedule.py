"""Time-step schedule of the reference's forward run, in the build's Real type.

Restates ``Glioma_ReactionDiffusion::run`` (Glioma/Glioma_ReactionDiffusion.cpp:
300-321):

* ``Dw = Dw / (L*L); Dg = 0.1 * Dw`` (``:302-303``), in Real;
* ``h = 1 / (blockSize * blocksPerDimension)`` (``:306``), the *initial-grid*
  spacing, in Real;
* ``dt = 0.99 * h*h / (2 * _DIM * max(Dw, Dg))`` (``:307``), evaluated in double
  and stored in Real;
* ``while (t <= tend) { step; t += dt; }`` with ``t`` a Real (``:317-321``).

``Real`` is float in the reference's default build (MRAG/MRAGcore/
MRAGCommon.h:43-47) and double in the FP64 build; both are supported here
with numpy scalars so every rounding matches.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

BLOCK_SIZE = 8
DIM = 3


def real_type(precision: str):
    if precision in ("f64", "double", "float64"):
        return np.float64
    if precision in ("f32", "float", "float32"):
        return np.float32
    raise ValueError(f"unknown precision {precision!r}")


@dataclass(frozen=True)
class Schedule:
    Dw: float      # rescaled white-matter diffusivity, as a Real
    Dg: float      # rescaled grey-matter diffusivity, as a Real
    rho: float     # proliferation rate, as a Real
    dt: float      # time step, as a Real (passed on as a double)
    nsteps: int    # iterations of the reference's while loop
    h: float       # initial-grid spacing
    precision: str


def make_schedule(Dw_cm2_day: float, rho_day: float, tend_day: float, L_cm: float,
                  blocks_per_dim: int, precision: str = "f64") -> Schedule:
    R = real_type(precision)
    Dw = R(Dw_cm2_day)
    rho = R(rho_day)
    tend = R(tend_day)
    L = R(L_cm)
    Dw = R(Dw / (L * L))
    Dg = R(0.1 * np.float64(Dw))
    h = R(1.0 / (BLOCK_SIZE * blocks_per_dim))
    mx = Dw if Dw >= Dg else Dg
    dt = R(0.99 * np.float64(h) * np.float64(h) / (2.0 * DIM * np.float64(mx)))
    t = R(0.0)
    n = 0
    while t <= tend:
        n += 1
        t = R(t + dt)
    return Schedule(float(Dw), float(Dg), float(rho), float(dt), n, float(h), precision)
