"""The C-ABI library loads and exports every symbol include/hpgb.h declares
(no GPU needed: nothing is computed)."""
import ctypes
import os
import re

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "hpgb.h")).read()
    return sorted(set(re.findall(r"HPGB_API\s+[\w\s\*]+?\b(hpgb_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "hpgb_create" in names and "hpgb_grid_visibilities" in names
    assert len(names) >= 25


def test_library_exports_every_declared_symbol(device_lib):
    lib = device_lib
    for name in declared_symbols():
        assert hasattr(lib, name), name
    assert lib.hpgb_abi_version() == 1


def test_python_binding_declares_every_symbol(device_lib):
    from hpg_b200 import abi
    assert set(declared_symbols()) <= set(abi.SIGNATURES)


def test_visdata_layout():
    """hpg::VisData<N> sizes (reference src/hpg.hpp:236-311)."""
    from hpg_b200 import visdata_dtype
    from oracle.oracle import visdata_dtype as odt
    for n, size in ((1, 88), (2, 96), (3, 112), (4, 120)):
        assert visdata_dtype(n).itemsize == size
        assert odt(n) == visdata_dtype(n)


def test_errors_without_device(device_lib):
    """Argument errors are values, not crashes, even with no GPU."""
    from hpg_b200 import abi
    lib = device_lib
    h = ctypes.c_void_p()
    gs = np.array([8, 8, 1, 1], np.uint32)
    sc = np.array([1.0, 1.0])
    m = np.array([0], np.int32)
    rc = lib.hpgb_create(0, 0, 1, abi.ptr(gs), abi.ptr(sc), 5, abi.ptr(m),
                         abi.ptr(m), ctypes.byref(h))
    assert rc == 1 + abi.ERROR_TYPES.index("InvalidNumberPolarizations")
    rc = lib.hpgb_fence(None)
    assert rc == 1 + abi.ERROR_TYPES.index("Other")
    assert lib.hpgb_last_error_message()
