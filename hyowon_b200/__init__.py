"""hyowon_b200 -- B200-native (sm_100a) particle-mesh gravity step and
kick-drift-kick update for the HYOWON cosmological N-body code.

The compute path is ``libhyowon_pm.so`` (hand-written CUDA + cuFFT) behind the
C ABI in ``include/hyowon_pm.h``; this package is the Python view of that ABI
and of the host-side cosmology scalars. Build with ``python -m hyowon_b200.build``.
"""
from .pm import (FP32_FIXED, FP64, CosmologyModel, DriftKickIntegrator,  # noqa: F401
                 LeapfrogIntegrator, MeshGeometry, PMForceMethod, PMSolver, TimeStep,
                 TimeStepper)
from ._native import (HyowonCudaError, HyowonLogicError,  # noqa: F401
                      HyowonUnderflowError, lib)

__all__ = [
    "FP64", "FP32_FIXED", "CosmologyModel", "DriftKickIntegrator", "LeapfrogIntegrator",
    "MeshGeometry", "PMForceMethod", "PMSolver", "TimeStep", "TimeStepper",
    "HyowonCudaError", "HyowonLogicError", "HyowonUnderflowError", "lib",
]
