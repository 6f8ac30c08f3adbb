"""soilb200: B200-native (sm_100a) Mobile V2 granular-terrain step.

Drop-in for the hot path of the reference project
wordxzl03-oss/Iron-soil-physical-simulation-algorithom-for-Isaac-Sim: the
Mobile V2 finite-volume step, MiniSlope repose relaxation and connected
large-avalanche (FailureZone) labelling, implemented as hand-written CUDA
kernels in ``libsoilb200.so`` behind a C ABI (``include/soilb200.h``).
"""

from ._lib import (  # noqa: F401
    B200BackendUnavailable,
    B200DeviceError,
    NumericalNonconvergenceError,
)
from .grid import DeviceGrid, choose_quantization  # noqa: F401
from .mobile_v2 import (  # noqa: F401
    B200MobileV2Solver,
    MobileV2Config,
    MobileV2State,
    MobileV2Step,
)

from .avalanche import (  # noqa: F401
    B200LargeAvalancheBridge,
    DeviceLargeAvalancheResult,
    LabelDiagnosis,
    LargeAvalancheTransitionConfig,
    MaterialScenario,
    label_mask,
    label_mask_preallocated,
    largest_connected_region,
)
from .relax import (  # noqa: F401
    EventDrivenMinimumSlopeAdapter,
    EventRelaxationResult,
    FrontierRelaxation,
    FrontierStats,
    MiniSlopeConfig,
    RelaxationStats,
    relax_critical_slope,
)

from .batch import B200PatchBatch  # noqa: E402,F401

# Reference-compatible aliases: code written against the reference's Warp
# device solver can switch by changing only the import.
WarpMobileV2ReferenceSolver = B200MobileV2Solver

__all__ = [
    "B200BackendUnavailable", "B200DeviceError", "NumericalNonconvergenceError",
    "DeviceGrid", "choose_quantization", "B200MobileV2Solver", "MobileV2Config",
    "MobileV2State", "MobileV2Step", "WarpMobileV2ReferenceSolver",
    "B200LargeAvalancheBridge", "LabelDiagnosis", "LargeAvalancheTransitionConfig",
    "MaterialScenario", "FrontierRelaxation", "FrontierStats", "RelaxationStats",
    "relax_critical_slope", "label_mask", "largest_connected_region",
    "label_mask_preallocated", "B200PatchBatch", "DeviceLargeAvalancheResult",
    "EventDrivenMinimumSlopeAdapter", "EventRelaxationResult", "MiniSlopeConfig",
]
