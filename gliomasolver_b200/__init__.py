"""gliomasolver_b200: GliomaSolver's Fisher-Kolmogorov RD hot path on B200.

The compute path is libgbfk.so (CUDA, sm_100a) behind the C ABI in
include/gbfk.h; this package is its host side: the ctypes binding, the
reference-shaped operator interface (``ReactionDiffusionOperator``,
``UpdateTumor``, ``BlockProcessing``), the time-step schedule of the
reference's driver and the seeded synthetic anatomy.
"""
from .schedule import Schedule, make_schedule  # noqa: F401
from ._lib import GbfkError  # noqa: F401
from .solver import (  # noqa: F401
    BlockPool,
    BlockProcessing,
    ReactionDiffusionOperator,
    UpdateTumor,
    reaction_diffusion_step,
)
