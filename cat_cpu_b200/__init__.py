"""cat_cpu_b200: B200-native Larger-than-Life stepping engine.

The compute path is libltl_b200.so (hand-written sm_100a CUDA behind a C ABI,
include/ltl.h); this package holds its sources (csrc/), the build script and a
ctypes host mirror of the reference's solver interface (ltl.py).
"""
from .ltl import (CASolverFactory, CUDASolver, Batch, LtlError, benchmark_seed, generate_state, start_grid,
                  compareCurrentStates, VARIANT_AUTO, VARIANT_PLAIN, VARIANT_TENSOR, VARIANT_PACKED,
                  VARIANT_NAMES, lib, pack_grid, unpack_grid)

__all__ = ["CASolverFactory", "CUDASolver", "Batch", "LtlError", "benchmark_seed", "generate_state", "start_grid",
           "compareCurrentStates", "VARIANT_AUTO", "VARIANT_PLAIN", "VARIANT_TENSOR", "VARIANT_PACKED",
           "VARIANT_NAMES", "lib", "pack_grid", "unpack_grid"]
