"""hpg_b200: B200-native (sm_100a) gridding and degridding for HPG.

The product is the CUDA library hpg_b200/lib/libhpgb.so behind the C ABI in
include/hpgb.h, the C++ hpg:: API in hpg_b200/cpp over that ABI, and this
Python binding (``Gridder``, mirroring hpg::Gridder).
"""
from .abi import (HpgError, device_count, load, visdata_dtype,  # noqa: F401
                  FFT_NEGATIVE, FFT_POSITIVE, SHIFT_BACKWARD, SHIFT_FORWARD,
                  PRECISION_FP64, PRECISION_MIXED)
from .gridder import (CFArray, Future, Gridder,  # noqa: F401
                      grid_visibilities_batch)

__all__ = ["HpgError", "device_count", "load", "visdata_dtype", "CFArray",
           "Future", "Gridder", "grid_visibilities_batch", "FFT_NEGATIVE", "FFT_POSITIVE",
           "SHIFT_BACKWARD", "SHIFT_FORWARD", "PRECISION_FP64",
           "PRECISION_MIXED"]
