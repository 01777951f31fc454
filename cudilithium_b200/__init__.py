"""cudilithium_b200: B200-native batched CRYSTALS-Dilithium (round 3, v3.1) engine.

The compute path is the CUDA library ``libcudilithium_b200.so`` (sm_100a kernels behind the C
ABI of ``include/cudilithium.h``); this package is its Python host side.  Importing it loads the
library and fails loudly if it is missing -- there is no CPU fallback.
"""
from ._lib import CudilError, lib, params  # noqa: F401
from .api import Dilithium, TaskLut, alloc_pool, ntt_mul, pinned  # noqa: F401

__all__ = ["Dilithium", "TaskLut", "CudilError", "alloc_pool", "ntt_mul", "pinned", "params", "lib"]
