"""CPU oracle for the windfvm CUDA library (test infrastructure only).

A C++ restatement of the reference's HLSL kernels (windfvm_oracle.cpp), loaded
through ctypes.  Only the tests, the smoke check and the benchmark's CPU
baseline use it; the library never does.
"""
from .binding import OracleSolver, build_oracle, log_law_wall_func

__all__ = ["OracleSolver", "build_oracle", "log_law_wall_func"]
