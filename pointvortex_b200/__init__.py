"""pointvortex_b200 — B200-native direct O(N^2) point-vortex velocity and RK4/DOPRI5 stepping.

The compute path is libpvb200.so (hand-written sm_100a CUDA behind the C ABI of
include/pvb200.h); this package is its host-side mirror of the reference's VelocityKernel
interface. Importing it without the built library raises ImportError.
"""
from .kernel import (  # noqa: F401
    CudaError,
    DeviceDipoleManager,
    DipoleEventState,
    DiskKernel,
    DipoleCandidate,
    InfinitePlaneKernel,
    Invariants,
    LogicError,
    PeriodicBoxKernel,
    StepResult,
    VelocityField,
    VelocityKernel,
    VortexSystem,
    backendName,
    backendRuntimeDetails,
    computeInvariants,
    makeBackendKernel,
    probePeak,
)
from ._lib import LIB_PATH  # noqa: F401
from . import autotune as _autotune

_autotune.load()  # the measured tuning table for this library, when present

__all__ = [
    "CudaError", "DeviceDipoleManager", "DipoleEventState", "DiskKernel", "DipoleCandidate", "InfinitePlaneKernel", "Invariants",
    "LogicError", "PeriodicBoxKernel", "StepResult", "VelocityField", "VelocityKernel",
    "VortexSystem", "backendName", "backendRuntimeDetails", "computeInvariants",
    "makeBackendKernel", "probePeak", "LIB_PATH",
]
