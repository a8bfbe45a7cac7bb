"""pencil_b200: the pencil FFT hot path of nogaki/pencil-rs on one B200.

Hand-written sm_100a kernels behind the C-ABI in ``include/pencil_b200.h``;
this package mirrors the reference's plan API over ctypes and adds
``torch.autograd`` wrappers built on the adjoint (VJP) kernels.
"""

from ._lib import InvalidSpectrum, PencilError, load  # noqa: F401
from .plans import (  # noqa: F401
    AllToAllvTransposePlan,
    C2cPlan,
    C2rPlan,
    DhtPlan,
    DistributedLayout,
    InPlaceArray,
    LocalTransposePlan,
    MixedC2cPlan,
    MixedR2cPlan,
    MpiTopology,
    Pencil,
    PlanBatch,
    R2cPlan,
    R2rPlan,
    SpatialRemapPlan,
    route_pencils,
)

__all__ = [
    "AllToAllvTransposePlan", "C2cPlan", "C2rPlan", "DhtPlan", "DistributedLayout", "InPlaceArray", "InvalidSpectrum",
    "LocalTransposePlan", "MixedC2cPlan", "MixedR2cPlan", "MpiTopology", "Pencil", "PencilError", "PlanBatch", "R2cPlan",
    "R2rPlan", "SpatialRemapPlan", "load", "route_pencils",
]
