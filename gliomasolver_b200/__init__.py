"""gliomasolver_b200: GliomaSolver's Fisher-Kolmogorov RD hot path on B200.

The compute path is libgbfk.so (CUDA, sm_100a) behind the C ABI in
include/gbfk.h; this package is its host side: the ctypes binding, the
reference-shaped operator interface (``ReactionDiffusionOperator``,
``UpdateTumor``, ``BlockProcessing``), the time-step schedule of the
reference's driver, the seeded synthetic anatomy, the patient data of the
reference (``patient``: Matrix files, anatomy and tumour mapping,
likelihood inputs), batched TMCMC stages and the TMCMC driver (``tmcmc``)
with the reference's TMCMC files (``tmcmc_io``), host snapshots of a pool so
that a long run can resume (``snapshot``), the adjoint as a
``torch.autograd.Function`` (``autograd``) and the sharding of a stage over
ranks (``shard``).
"""
from . import patient  # noqa: F401
from . import snapshot  # noqa: F401
from .schedule import Schedule, make_schedule  # noqa: F401
from ._lib import GbfkError  # noqa: F401
from .solver import (  # noqa: F401
    BlockPool,
    BlockProcessing,
    ReactionDiffusionOperator,
    UpdateTumor,
    reaction_diffusion_step,
)
