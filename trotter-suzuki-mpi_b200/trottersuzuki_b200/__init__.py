"""B200-native Trotter-Suzuki evolution (drop-in for trotter-suzuki-mpi's evolution path).

Low level: `Kernel` (one tile on the GPU, C ABI in include/ts_b200.h).
"""
from .kernel import FP32, FP64, Kernel, launch_count, version  # noqa: F401
from ._capi import B200Error, Desc, EnergyParams  # noqa: F401

__version__ = "1.6.2+b200"
