"""e8qlib on B200: the E8Q IVF index with its search path on the GPU (sm_100a).

Drop-in for the reference package's ``E8qIndex`` and ``Me8qIndex`` (same
constructors, methods, argument names, dtypes, shapes and exceptions). The compiled pieces live next
to this file: ``libe8qcuda.so`` (CUDA kernels behind the C ABI in
include/e8qc.h) and ``_e8qlib`` (the pybind11 module over it). Importing fails
loudly when they are missing; there is no CPU path.
"""
from ._e8qlib import (E8qIndex, Me8qIndex, Plan, Server, branch_levels, debug_fail_host_allocs, encode,  # noqa: F401
                      fixed_scale, rotate, tc_i8_gemm, version)

__all__ = ["E8qIndex", "Me8qIndex", "Plan", "Server", "branch_levels", "debug_fail_host_allocs", "encode", "fixed_scale",
           "rotate", "tc_i8_gemm", "version"]
