"""incrmt_b200: a B200-native implementation of IncRMT's per-timestep hot path.

The compute path is libincrmt_gpu.so (hand-written sm_100a CUDA behind the C
ABI declared in include/incrmt.h). This package binds that ABI with ctypes.
There is no CPU fallback: importing the binding fails loudly when the library
has not been built (python -m incrmt_b200.build).
"""
from . import capi  # noqa: F401
from .capi import (  # noqa: F401
    IncrmtError, MGSolver, SYS_MAC, SYS_FEM, PREC_FP64, PREC_MIXED, lib_path,
)
