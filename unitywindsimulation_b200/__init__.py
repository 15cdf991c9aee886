"""B200-native urban-wind FVM solver (drop-in for the HLSL dispatch path of
puppy2333/UnityWindSimulation).  Compute lives in libwindfvm.so (C ABI,
include/windfvm.h); this package is the host-side mirror of the reference's
IFvmSolver interface plus the seeded case generator."""
from . import _lib
from ._lib import WfConfig, WindFvmError
from .config import default_config
from .solver import FvmSolverCuda, FvmSolverGpu

__all__ = ["FvmSolverCuda", "FvmSolverGpu", "WfConfig", "WindFvmError", "default_config", "_lib"]
