"""ctypes binding of libhpgb.so (include/hpgb.h).

This is the Python side of the C ABI: it loads the in-tree sm_100a library,
declares every entry point, maps status codes to ``HpgError`` and provides the
numpy record types of ``hpg::VisData<N>`` (reference src/hpg.hpp:236-311).
It never falls back to anything else: if the library is missing,
``load()`` raises.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libhpgb.so")

# hpg::ErrorType (reference src/hpg_error.hpp:26-38); status = 1 + value
ERROR_TYPES = [
    "DisabledDevice",
    "DisabledHostDevice",
    "OutOfBoundsCFIndex",
    "InvalidNumberMuellerIndexRows",
    "InvalidNumberPolarizations",
    "InvalidCFLayout",
    "InvalidModelGridSize",
    "ExcessiveNumberVisibilities",
    "UpdateWeightsWithoutGridding",
    "CFSupportExceedsGrid",
    "Other",
]

UPDATE_GRID_WEIGHTS = 1
DO_DEGRID = 2
RETURN_VISIBILITIES = 4
DO_GRID = 8

LAYOUT_RIGHT = 0
LAYOUT_LEFT = 1

FFT_POSITIVE = 0
FFT_NEGATIVE = 1

SHIFT_FORWARD = 0
SHIFT_BACKWARD = 1

PRECISION_FP64 = 0
PRECISION_MIXED = 1

KERNEL_AUTO = 0
KERNEL_DIRECT = 1
KERNEL_TILED = 2

CF_LAYOUT_LOGICAL = 0
CF_LAYOUT_CUDA_V0 = 1
CF_LAYOUT_HOST_V0 = 2

# capacity of the fixed scratch array of hpgb_grid_visibilities_noalloc
NOALLOC_MAX_VALUES = 1048576


class HpgError(RuntimeError):
    """A failed C-ABI call; ``type`` is the hpg::ErrorType name."""

    def __init__(self, code, message):
        self.code = code
        self.type = ERROR_TYPES[code - 1] if 1 <= code <= len(ERROR_TYPES) else "Other"
        super().__init__(f"{self.type}: {message}")


def visdata_dtype(npol):
    """numpy dtype with the exact layout of hpg::VisData<npol>."""
    if npol not in (1, 2, 3, 4):
        raise ValueError("npol must be 1..4")
    off_w = 8 * npol
    off_freq = (12 * npol + 7) // 8 * 8
    return np.dtype({
        "names": ["vis", "weights", "freq", "phase", "uvw", "grid_cube",
                  "cf_index", "cf_phase_gradient"],
        "formats": [(np.complex64, (npol,)), (np.float32, (npol,)), np.float64,
                    np.float64, (np.float64, (3,)), np.uint32,
                    (np.uint32, (2,)), (np.float64, (2,))],
        "offsets": [0, off_w, off_freq, off_freq + 8, off_freq + 16,
                    off_freq + 40, off_freq + 44, off_freq + 56],
        "itemsize": off_freq + 72,
    })


COORDS_DTYPE = np.dtype([
    ("grid_coord", np.int32, (2,)), ("cf_major", np.int32, (2,)),
    ("cf_minor", np.int32, (2,)), ("fine_offset", np.int32, (2,)),
    ("cf_size", np.int32, (2,)), ("pos_w", np.int32), ("in_grid", np.int32),
    ("grid_mueller", np.int32, (4, 4)), ("degrid_mueller", np.int32, (4, 4))])

_lib = None

_P = ctypes.c_void_p
_PP = ctypes.POINTER(ctypes.c_void_p)
_U = ctypes.c_uint
_I = ctypes.c_int
_S = ctypes.c_size_t
_D = ctypes.c_double

SIGNATURES = {
    "hpgb_abi_version": ([], _I),
    "hpgb_last_error_message": ([], ctypes.c_char_p),
    "hpgb_device_count": ([ctypes.POINTER(_I)], _I),
    "hpgb_create": ([_I, _U, _S, _P, _P, _U, _P, _P, _PP], _I),
    "hpgb_clone": ([_P, _PP], _I),
    "hpgb_destroy": ([_P], _I),
    "hpgb_set_precision": ([_P, _I], _I),
    "hpgb_set_gridding_kernel": ([_P, _I], _I),
    "hpgb_get_stream": ([_P, _PP], _I),
    "hpgb_cf_region_size": ([_P, _U, _U, _P, ctypes.POINTER(_S)], _I),
    "hpgb_allocate_cf_region": ([_P, _U, _U, _P], _I),
    "hpgb_set_cf": ([_P, _U, _U, _P, _PP, _I, _I], _I),
    "hpgb_set_model": ([_P, _P, _P, _I, _I], _I),
    "hpgb_grid_visibilities": ([_P, _P, _S, _U, _U, _I, _P], _I),
    "hpgb_grid_visibilities_noalloc": ([_P, _P, _S, _U, _U], _I),
    "hpgb_degrid_linear": ([_P, _P, _S, _U, _P, _P], _I),
    "hpgb_degrid_adjoint": ([_P, _P, _S, _U, _P, _P], _I),
    "hpgb_grid_linear": ([_P, _P, _S, _U, _P, _P], _I),
    "hpgb_grid_adjoint": ([_P, _P, _S, _U, _P, _P], _I),
    "hpgb_fence": ([_P], _I),
    "hpgb_copy_weights": ([_P, _P, _I], _I),
    "hpgb_copy_grid": ([_P, _P, _I], _I),
    "hpgb_copy_model": ([_P, _P, _I], _I),
    "hpgb_weights_device_ptr": ([_P, _PP, ctypes.POINTER(_S)], _I),
    "hpgb_grid_device_ptr": ([_P, _PP, ctypes.POINTER(_S)], _I),
    "hpgb_model_device_ptr": ([_P, _PP, ctypes.POINTER(_S)], _I),
    "hpgb_reset_grid": ([_P], _I),
    "hpgb_reset_model": ([_P], _I),
    "hpgb_normalize_by_weights": ([_P, _D], _I),
    "hpgb_apply_grid_fft": ([_P, _D, _I, _I], _I),
    "hpgb_apply_model_fft": ([_P, _D, _I, _I], _I),
    "hpgb_image_grid": ([_P, _D, _D, _I, _I], _I),
    "hpgb_shift_grid": ([_P, _I], _I),
    "hpgb_shift_model": ([_P, _I], _I),
    "hpgb_kernel_launches": ([_P, ctypes.POINTER(ctypes.c_uint64)], _I),
    "hpgb_set_tiled_plan": ([_P, _I, _I], _I),
    "hpgb_last_gridding_kernel": ([_P, ctypes.POINTER(ctypes.c_int)], _I),
    "hpgb_set_tiled_plan_ex": ([_P, ctypes.c_void_p], _I),
    "hpgb_set_wait_limit": ([_P, ctypes.c_double], _I),
    "hpgb_grid_visibilities_batch": ([_P, ctypes.c_size_t, _P, _P, ctypes.c_uint,
                                      ctypes.c_uint, _I, _P], _I),
    "hpgb_debug_withhold_copy": ([_P, ctypes.c_longlong], _I),
    "hpgb_get_tiled_plan": ([_P, ctypes.c_void_p], _I),
    "hpgb_autotune_tiled": ([_P, _P, _S, _U, _U, _I, ctypes.POINTER(_I),
                             ctypes.POINTER(_I)], _I),
    "hpgb_begin_capture": ([_P], _I),
    "hpgb_end_capture": ([_P, _PP], _I),
    "hpgb_graph_launch": ([_P, _P], _I),
    "hpgb_graph_destroy": ([_P], _I),
    "hpgb_profile_tiled_kernel": ([_P, _I], _I),
    "hpgb_tiled_kernel_time": ([_P, ctypes.POINTER(_D),
                                ctypes.POINTER(ctypes.c_uint64)], _I),
    "hpgb_debug_coords": ([_P, _P, _S, _U, _P], _I),
}


class TiledPlan(ctypes.Structure):
    """hpgb_tiled_plan (include/hpgb.h): 0 in a field = automatic."""
    _fields_ = [("ring_parts", ctypes.c_int), ("chunk_vis", ctypes.c_int),
                ("tile_side", ctypes.c_int), ("compensated", ctypes.c_int)]


COMPENSATED_OFF = 1
COMPENSATED_ON = 2


def load(path=LIB_PATH):
    """Load libhpgb.so and declare its entry points (cached)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(
            f"{path} not found: build the CUDA library first "
            "(python -m hpg_b200.build); there is no CPU fallback")
    lib = ctypes.CDLL(path)
    for name, (args, res) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    if lib.hpgb_abi_version() != 1:
        raise ImportError("libhpgb.so ABI version mismatch")
    _lib = lib
    return lib


def check(code):
    if code != 0:
        msg = load().hpgb_last_error_message().decode()
        raise HpgError(code, msg)


def ptr(a):
    """Address of a contiguous numpy array, or of a torch tensor."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return ctypes.c_void_p(a.data_ptr())
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be C-contiguous")
    return ctypes.c_void_p(a.ctypes.data)


def device_count():
    c = _I(0)
    check(load().hpgb_device_count(ctypes.byref(c)))
    return c.value
