"""cms2d_b200: B200-native (sm_100a) implicit hot path of CMS-Flow.

The compute path is libcmsgpu.so (hand-written CUDA kernels + a C-ABI, see
include/cmsgpu.h); the Python modules here mirror the reference's interfaces
on top of it and generate synthetic grids.
"""
from . import grid  # noqa: F401
from . import solver  # noqa: F401

__all__ = ["grid", "solver"]
__version__ = "0.1.0"
