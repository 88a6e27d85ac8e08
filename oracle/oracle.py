"""ctypes wrapper of the CPU oracle (oracle/hpg_oracle.cc).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the product package.

Arrays follow the same conventions as the product binding: grids complex128
(cube, mrow, y, x), weights float64 (cube, mrow), visibilities are record
arrays with the byte layout of hpg::VisData<N> (reference src/hpg.hpp:236-311),
CF groups complex64 in the CFArray logical order (x, y, mueller, cube).
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")


def build():
    """Compile liboracle.so with the recipe in oracle/Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return LIB_PATH


def visdata_dtype(npol):
    off_freq = (12 * npol + 7) // 8 * 8
    return np.dtype({
        "names": ["vis", "weights", "freq", "phase", "uvw", "grid_cube",
                  "cf_index", "cf_phase_gradient"],
        "formats": [(np.complex64, (npol,)), (np.float32, (npol,)), np.float64,
                    np.float64, (np.float64, (3,)), np.uint32,
                    (np.uint32, (2,)), (np.float64, (2,))],
        "offsets": [0, 8 * npol, off_freq, off_freq + 8, off_freq + 16,
                    off_freq + 40, off_freq + 44, off_freq + 56],
        "itemsize": off_freq + 72,
    })


class _Params(ctypes.Structure):
    _fields_ = [
        ("grid_size", ctypes.c_int * 4),
        ("grid_scale", ctypes.c_double * 2),
        ("npol", ctypes.c_int),
        ("mueller", (ctypes.c_int * 4) * 4),
        ("conj_mueller", (ctypes.c_int * 4) * 4),
        ("oversampling", ctypes.c_int),
        ("ngroups", ctypes.c_int),
        ("cf_extents", ctypes.POINTER(ctypes.c_uint)),
        ("cf_values", ctypes.POINTER(ctypes.c_void_p)),
    ]


COORDS_DTYPE = np.dtype([
    ("grid_coord", np.int32, (2,)), ("cf_major", np.int32, (2,)),
    ("cf_minor", np.int32, (2,)), ("fine_offset", np.int32, (2,)),
    ("cf_size", np.int32, (2,)), ("pos_w", np.int32), ("in_grid", np.int32),
    ("grid_mueller", np.int32, (4, 4)), ("degrid_mueller", np.int32, (4, 4))])

_lib = None


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        lib = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        lib.oracle_num_threads.restype = ctypes.c_int
        lib.oracle_vis_coords.argtypes = [P, P, ctypes.c_size_t, ctypes.c_int, P]
        lib.oracle_normalisers.argtypes = [P, P, ctypes.c_size_t, ctypes.c_int, P]
        lib.oracle_grid_visibilities.argtypes = [
            P, P, ctypes.c_size_t, ctypes.c_int, ctypes.c_int, ctypes.c_int,
            ctypes.c_int, ctypes.c_int, P, P, P, ctypes.c_int]
        lib.oracle_normalize_by_weights.argtypes = [P, P, P, ctypes.c_double]
        lib.oracle_normalize.argtypes = [P, P, ctypes.c_double]
        lib.oracle_shift.argtypes = [P, P, ctypes.c_int]
        lib.oracle_cone_cf.argtypes = [ctypes.c_uint, ctypes.c_uint,
                                       ctypes.c_uint, P]
        _lib = lib
    return _lib


def num_threads():
    return load().oracle_num_threads()


def _ptr(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


class Oracle:
    """CPU restatement of one gridder: same state as hpg::GridderState."""

    def __init__(self, grid_size, grid_scale, mueller_indexes,
                 conjugate_mueller_indexes, oversampling, cf_extents,
                 cf_values):
        self.grid_size = tuple(int(x) for x in grid_size)
        self.npol = len(mueller_indexes[0])
        nx, ny, nr, nc = self.grid_size
        self.grid = np.zeros((nc, nr, ny, nx), np.complex128)
        self.weights = np.zeros((nc, nr), np.float64)
        self.model = None
        p = _Params()
        for i in range(4):
            p.grid_size[i] = self.grid_size[i]
        p.grid_scale[0], p.grid_scale[1] = grid_scale
        p.npol = self.npol
        for r in range(4):
            for c in range(4):
                p.mueller[r][c] = (mueller_indexes[r][c]
                                   if r < len(mueller_indexes) and c < self.npol else -1)
                p.conj_mueller[r][c] = (conjugate_mueller_indexes[r][c]
                                        if r < len(conjugate_mueller_indexes)
                                        and c < self.npol else -1)
        p.oversampling = int(oversampling)
        p.ngroups = len(cf_extents)
        self._ext = np.ascontiguousarray(np.asarray(cf_extents, np.uint32).reshape(-1))
        self._vals = [np.ascontiguousarray(v, np.complex64) for v in cf_values]
        self._vptr = (ctypes.c_void_p * max(len(self._vals), 1))(
            *[v.ctypes.data for v in self._vals])
        p.cf_extents = self._ext.ctypes.data_as(ctypes.POINTER(ctypes.c_uint))
        p.cf_values = ctypes.cast(self._vptr, ctypes.POINTER(ctypes.c_void_p))
        self._p = p
        self._gs = np.asarray(self.grid_size, np.int32)

    def set_model(self, model):
        self.model = None if model is None else np.ascontiguousarray(model, np.complex128)

    def vis_coords(self, vis):
        vis = np.ascontiguousarray(vis)
        out = np.zeros(len(vis), COORDS_DTYPE)
        rc = load().oracle_vis_coords(ctypes.byref(self._p), _ptr(vis), len(vis),
                                      self.npol, _ptr(out))
        assert rc == 0
        return out

    def normalisers(self, vis):
        """Degridding normaliser per visibility polarization (reference
        src/hpg_core.hpp:598-600, :659-661), complex128 [n][npol]."""
        vis = np.ascontiguousarray(vis)
        out = np.zeros((len(vis), self.npol), np.complex128)
        rc = load().oracle_normalisers(ctypes.byref(self._p), _ptr(vis),
                                       len(vis), self.npol, _ptr(out))
        assert rc == 0
        return out

    def grid_visibilities(self, vis, update_weights=True, do_degrid=False,
                          return_vis=False, do_grid=True, nthreads=1):
        """One VisibilityGridder<N>::kernel call (reference
        src/hpg_core.hpp:1082-1253).  Returns the updated visibility array
        when return_vis is set."""
        vis = np.array(vis, copy=True)
        rc = load().oracle_grid_visibilities(
            ctypes.byref(self._p), _ptr(vis), len(vis), self.npol,
            int(update_weights), int(do_degrid), int(return_vis), int(do_grid),
            _ptr(self.grid), _ptr(self.weights), _ptr(self.model), int(nthreads))
        assert rc == 0
        return vis if return_vis else None

    def normalize_by_weights(self, wfactor=1.0):
        load().oracle_normalize_by_weights(_ptr(self.grid), _ptr(self.weights),
                                           _ptr(self._gs), float(wfactor))

    def normalize(self, norm):
        load().oracle_normalize(_ptr(self.grid), _ptr(self._gs), float(norm))

    def shift_grid(self, direction):
        load().oracle_shift(_ptr(self.grid), _ptr(self._gs), int(direction))


def fft_grid(grid, sign_positive=True):
    """2-D FFT of every (cube, mrow) plane of a (cube, mrow, y, x) grid with
    the reference's sign convention (src/hpg_core.hpp:2069, :2166): POSITIVE
    is the unnormalised inverse transform, NEGATIVE the forward transform."""
    if sign_positive:
        ny, nx = grid.shape[-2:]
        return np.fft.ifft2(grid, axes=(-2, -1)) * (nx * ny)
    return np.fft.fft2(grid, axes=(-2, -1))


def cone_cf(nmueller, oversampling, radius):
    """ConeCFArray of the reference's tests (GridderStateUnitTests.cc:198-259),
    one group, complex64 (x, y, mueller, cube=1); computed with glibc float
    math like the reference's fixture."""
    w = 2 * (radius + 2) * oversampling + 1
    out = np.zeros((w, w, nmueller, 1), np.complex64)
    load().oracle_cone_cf(nmueller, oversampling, radius, _ptr(out))
    return out
