"""B200-native compressible RHS + SSP-RK stage update for madvait/Chimera_Comp_LES.

The product is ``libchimera_b200.so`` (sm_100a CUDA kernels behind the C-ABI in
``include/chimera_b200.h``); ``Block`` mirrors the reference's hot-path calls
over that C-ABI.
"""
from ._lib import CB_FP64, CB_MIXED, IBM_INFO_DTYPE, ChimeraError, LIB_PATH, load  # noqa: F401
from .solver import Block  # noqa: F401
from . import workloads  # noqa: F401

__all__ = ["Block", "ChimeraError", "load", "LIB_PATH", "workloads"]
