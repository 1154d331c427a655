"""emergence_b200: B200-native (sm_100a) compressible-Euler step.

Drop-in for the explicit finite-volume step of the emergence workspace's
``compressible`` crate (WCNS WENO5-Z reconstruction, HLLC, positivity
limiter, SSP-RK3, ghost fill, CFL reduction), behind the C ABI of
``include/emergence_b200.h``.
"""
from .physics import Bc, Euler, FluxMode, Mesh, Nasg, Precision, initial_state
from .solver import GpuSolver, device_count, release_memory, state_hash
from .amr import GpuAmr
from .batch import GpuBatch1D
from .adjoint import DifferentiableSolver
from .five import FiveEq, GpuFiveSolver, five_initial_state
from ._abi import EmgError, LIB_PATH

__all__ = ["Bc", "Euler", "FluxMode", "Mesh", "Nasg", "Precision", "initial_state", "GpuSolver", "GpuAmr", "GpuBatch1D", "DifferentiableSolver", "FiveEq", "GpuFiveSolver", "five_initial_state", "device_count", "release_memory", "state_hash",
           "EmgError", "LIB_PATH"]
