"""espec_b200 -- B200-native (sm_100a) propagation path of eSPec.

The product is the CUDA library libespecgpu.so (espec_b200/csrc, C-ABI in
include/espec_gpu.h).  This package is its host-side mirror: ctypes bindings
and the batched split-operator interface.
"""
from . import _native
from ._native import EspecError, load
from .grid import PsodGrid, SilGrid, SodGrid, SpoGrid
from .spo import SodBatch, SpoBatch

__all__ = ["EspecError", "PsodGrid", "SilGrid", "SodGrid", "SpoGrid", "SodBatch", "SpoBatch", "load", "workloads"]
