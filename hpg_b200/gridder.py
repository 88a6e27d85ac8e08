"""Python mirror of the reference's hpg::Gridder / hpg::GridderState API
(reference src/hpg.hpp:1103-2795, src/hpg.cc:974-1400) over the C ABI.

Method names, argument meaning, defaults and error behaviour follow the
reference; errors are raised as ``HpgError`` whose ``type`` is the
hpg::ErrorType name.  Arrays use numpy shapes in the reference's device
layout: grids are complex128 ``(cube, mrow, y, x)`` (LayoutLeft
[x, y, mrow, cube]), weights are float64 ``(cube, mrow)``, visibilities are
``visdata_dtype(npol)`` record arrays.  Torch CUDA tensors are accepted
wherever ``on_device=True`` is given.
"""
import ctypes

import numpy as np

from . import abi
from .abi import HpgError, check, load, ptr, visdata_dtype

# hpg::CFArray::padding (reference src/hpg.hpp:655)
CF_PADDING = 2


class CFArray:
    """Convolution function values for the C ABI.

    ``values[g]`` holds group g as complex64 in the CFArray logical index
    order (x, y, mueller, cube), i.e. a C-contiguous array of shape
    ``extents[g]`` (reference src/hpg.hpp:646-721); ``layout`` may instead
    name one of the reference's device layouts ("0-Cuda", "0-Serial",
    "0-OpenMP"), in which case ``values[g]`` is that flat buffer.
    """

    def __init__(self, oversampling, extents, values, layout=None):
        self.oversampling = int(oversampling)
        self.extents = [tuple(int(e) for e in ext) for ext in extents]
        self.values = list(values)
        self.layout = layout

    def num_groups(self):
        return len(self.extents)

    def radii(self, grp):
        # reference src/hpg.hpp:687-694
        os_ = self.oversampling
        ext = self.extents[grp]
        return (((ext[0] - 2 * CF_PADDING * os_) // os_) // 2,
                ((ext[1] - 2 * CF_PADDING * os_) // os_) // 2)

    def layout_code(self):
        if self.layout in (None, "logical"):
            return abi.CF_LAYOUT_LOGICAL
        if self.layout == "0-Cuda":
            return abi.CF_LAYOUT_CUDA_V0
        if self.layout in ("0-Serial", "0-OpenMP"):
            return abi.CF_LAYOUT_HOST_V0
        raise HpgError(abi.ERROR_TYPES.index("InvalidCFLayout") + 1,
                       f"unsupported CF layout {self.layout!r}")


class Future:
    """Value resolved at the next fence (reference hpg::future,
    src/hpg.hpp:1004-1066): ``get()`` returns None until then."""

    def __init__(self, gridder, value):
        self._gridder = gridder
        self._value = value
        self._epoch = gridder._fence_epoch

    def get(self):
        if self._gridder._fence_epoch > self._epoch:
            return self._value
        return None


class Gridder:
    """Mutable gridder on the B200 device (reference hpg::Gridder)."""

    def __init__(self, handle, npol, grid_size, grid_scale, max_batch,
                 max_added_tasks):
        self._h = handle
        self.npol = npol
        self.grid_size = tuple(grid_size)
        self.grid_scale = tuple(grid_scale)
        self.max_visibility_batch_size = max_batch
        self.max_added_tasks = max_added_tasks
        self._fence_epoch = 0

    # -- construction -------------------------------------------------------

    @classmethod
    def create(cls, device=0, max_added_tasks=0, max_visibility_batch_size=1,
               init_cf_shape=None, grid_size=(1, 1, 1, 1),
               grid_scale=(1.0, 1.0), mueller_indexes=((0,),),
               conjugate_mueller_indexes=((0,),)):
        """GridderState::create (reference src/hpg.cc:226-264)."""
        lib = load()
        gs = np.asarray(grid_size, dtype=np.uint32)
        if len(gs) != 4:
            raise ValueError("grid_size has four axes: x, y, mrow, cube")
        mi = [list(r) for r in mueller_indexes]
        ci = [list(r) for r in conjugate_mueller_indexes]
        if gs[2] != len(mi) or gs[2] != len(ci):
            raise HpgError(4, "Number of rows of Mueller indexes does not "
                              "match grid")
        npol = len(mi[0]) if mi else 0
        m = np.asarray(mi, dtype=np.int32).reshape(-1)
        c = np.asarray(ci, dtype=np.int32).reshape(-1)
        sc = np.asarray(grid_scale, dtype=np.float64)
        h = ctypes.c_void_p()
        check(lib.hpgb_create(int(device), int(max_added_tasks),
                              int(max_visibility_batch_size), ptr(gs),
                              ptr(sc), npol, ptr(m), ptr(c), ctypes.byref(h)))
        g = cls(h, npol, [int(x) for x in gs], [float(x) for x in sc],
                int(max_visibility_batch_size), int(max_added_tasks))
        if init_cf_shape is not None:
            g.allocate_convolution_function_region(init_cf_shape)
        return g

    def copy(self):
        """Deep copy (GridderState copy constructor, src/hpg.cc:266-268)."""
        h = ctypes.c_void_p()
        check(load().hpgb_clone(self._h, ctypes.byref(h)))
        g = Gridder(h, self.npol, self.grid_size, self.grid_scale,
                    self.max_visibility_batch_size, self.max_added_tasks)
        return g

    def close(self):
        if self._h:
            check(load().hpgb_destroy(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def is_null(self):
        return not self._h

    def num_polarizations(self):
        return self.npol

    # -- configuration ------------------------------------------------------

    def set_precision(self, precision):
        check(load().hpgb_set_precision(self._h, int(precision)))

    def set_gridding_kernel(self, kind):
        """abi.KERNEL_AUTO, KERNEL_DIRECT or KERNEL_TILED."""
        check(load().hpgb_set_gridding_kernel(self._h, int(kind)))

    @property
    def stream(self):
        s = ctypes.c_void_p()
        check(load().hpgb_get_stream(self._h, ctypes.byref(s)))
        return s.value

    @staticmethod
    def _extents(shape):
        ext = np.asarray([list(e) for e in shape.extents], dtype=np.uint32)
        return ext.reshape(-1), len(shape.extents)

    def convolution_function_region_size(self, shape):
        n = ctypes.c_size_t()
        if shape is None:
            check(load().hpgb_cf_region_size(self._h, 0, 0, None, ctypes.byref(n)))
        else:
            ext, ng = self._extents(shape)
            check(load().hpgb_cf_region_size(self._h, shape.oversampling, ng,
                                             ptr(ext), ctypes.byref(n)))
        return n.value

    def allocate_convolution_function_region(self, shape):
        ext, ng = self._extents(shape)
        check(load().hpgb_allocate_cf_region(self._h, shape.oversampling, ng,
                                             ptr(ext)))

    def set_convolution_function(self, cf, on_device=False):
        """GridderState::set_convolution_function (src/hpg.cc:381-408)."""
        ext, ng = self._extents(cf)
        layout = cf.layout_code()
        keep = []
        arr = (ctypes.c_void_p * max(ng, 1))()
        for g in range(ng):
            v = cf.values[g]
            if not on_device:
                v = np.ascontiguousarray(v, dtype=np.complex64)
            keep.append(v)
            arr[g] = ptr(v).value
        check(load().hpgb_set_cf(self._h, cf.oversampling, ng, ptr(ext),
                                 ctypes.cast(arr, ctypes.POINTER(ctypes.c_void_p)),
                                 layout, 1 if on_device else 0))

    def set_model(self, values, layout="left", on_device=False):
        """GridderState::set_model (src/hpg.cc:409-432).  ``values`` is
        complex128 of shape (cube, mrow, y, x) for layout "left", or
        (x, y, mrow, cube) for layout "right"."""
        if layout == "left":
            code = abi.LAYOUT_LEFT
            ext = np.asarray(values.shape[::-1], dtype=np.uint32)
        else:
            code = abi.LAYOUT_RIGHT
            ext = np.asarray(values.shape, dtype=np.uint32)
        if not on_device:
            values = np.ascontiguousarray(values, dtype=np.complex128)
        check(load().hpgb_set_model(self._h, ptr(values), ptr(ext), code,
                                    1 if on_device else 0))

    # -- gridding -----------------------------------------------------------

    def _grid(self, vis, flags, on_device, npol=None):
        npol = self.npol if npol is None else npol
        if on_device:
            n = vis.numel() * vis.element_size() // abi.visdata_dtype(npol).itemsize
            out = vis if flags & abi.RETURN_VISIBILITIES else None
            check(load().hpgb_grid_visibilities(self._h, ptr(vis), n, npol,
                                                flags, 1, ptr(out)))
            return out
        vis = np.ascontiguousarray(vis)
        out = None
        if flags & abi.RETURN_VISIBILITIES:
            out = np.empty_like(vis)
        check(load().hpgb_grid_visibilities(self._h, ptr(vis), len(vis), npol,
                                            flags, 0, ptr(out)))
        return out

    def grid_visibilities(self, visibilities, update_grid_weights=True,
                          on_device=False):
        """reference src/hpg.cc:493-496: (w, F, F, T)"""
        flags = abi.DO_GRID | (abi.UPDATE_GRID_WEIGHTS if update_grid_weights else 0)
        self._grid(visibilities, flags, on_device)

    def degrid_grid_visibilities(self, visibilities, update_grid_weights=True,
                                 on_device=False):
        """reference src/hpg.cc:537-540: (w, T, F, T)"""
        flags = abi.DO_DEGRID | abi.DO_GRID | (
            abi.UPDATE_GRID_WEIGHTS if update_grid_weights else 0)
        self._grid(visibilities, flags, on_device)

    def degrid_get_predicted_visibilities(self, visibilities, on_device=False):
        """reference src/hpg.cc:577-583: (F, T, T, F); returns a Future."""
        out = self._grid(visibilities, abi.DO_DEGRID | abi.RETURN_VISIBILITIES,
                         on_device)
        return Future(self, out)

    def degrid_grid_get_residual_visibilities(self, visibilities,
                                              update_grid_weights=True,
                                              on_device=False):
        """reference src/hpg.cc:612-619: (w, T, T, T); returns a Future."""
        flags = (abi.DO_DEGRID | abi.DO_GRID | abi.RETURN_VISIBILITIES |
                 (abi.UPDATE_GRID_WEIGHTS if update_grid_weights else 0))
        out = self._grid(visibilities, flags, on_device)
        return Future(self, out)

    def raw_grid_visibilities(self, visibilities, flags, on_device=False,
                              npol=None):
        """State::grid_visibilities with explicit flags (validation order of
        src/hpg_runtime.hpp:1816-1828 applies)."""
        return self._grid(visibilities, flags, on_device, npol)

    def fence(self):
        check(load().hpgb_fence(self._h))
        self._fence_epoch += 1

    # -- results ------------------------------------------------------------

    def grid_weights(self, layout="left"):
        nx, ny, nr, nc = self.grid_size
        code = abi.LAYOUT_LEFT if layout == "left" else abi.LAYOUT_RIGHT
        out = np.empty((nc, nr) if layout == "left" else (nr, nc), np.float64)
        check(load().hpgb_copy_weights(self._h, ptr(out), code))
        self._fence_epoch += 1
        return out

    def _values(self, fn, layout):
        nx, ny, nr, nc = self.grid_size
        code = abi.LAYOUT_LEFT if layout == "left" else abi.LAYOUT_RIGHT
        shape = (nc, nr, ny, nx) if layout == "left" else (nx, ny, nr, nc)
        out = np.empty(shape, np.complex128)
        check(fn(self._h, ptr(out), code))
        self._fence_epoch += 1
        return out

    def grid_values(self, layout="left"):
        return self._values(load().hpgb_copy_grid, layout)

    def model_values(self, layout="left"):
        return self._values(load().hpgb_copy_model, layout)

    def _device_ptr(self, fn):
        p = ctypes.c_void_p()
        n = ctypes.c_size_t()
        check(fn(self._h, ctypes.byref(p), ctypes.byref(n)))
        return p.value, n.value

    def grid_values_ptr(self):
        return self._device_ptr(load().hpgb_grid_device_ptr)

    def grid_weights_ptr(self):
        return self._device_ptr(load().hpgb_weights_device_ptr)

    def model_values_ptr(self):
        return self._device_ptr(load().hpgb_model_device_ptr)

    def image_grid(self, wfactor=1.0, norm=1.0, sign=None, direction=None):
        """normalize_by_weights(wfactor), apply_grid_fft(norm, sign) and
        shift_grid(direction) as one FFT and one pass over the grid."""
        sign = abi.FFT_POSITIVE if sign is None else int(sign)
        direction = abi.SHIFT_FORWARD if direction is None else int(direction)
        check(load().hpgb_image_grid(self._h, float(wfactor), float(norm),
                                     sign, direction))

    def reset_grid(self):
        check(load().hpgb_reset_grid(self._h))

    def reset_model(self):
        check(load().hpgb_reset_model(self._h))

    def normalize_by_weights(self, wgt_factor=1.0):
        check(load().hpgb_normalize_by_weights(self._h, float(wgt_factor)))

    def apply_grid_fft(self, norm=1.0, sign=abi.FFT_POSITIVE, in_place=True):
        check(load().hpgb_apply_grid_fft(self._h, float(norm), int(sign),
                                         1 if in_place else 0))

    def apply_model_fft(self, norm=1.0, sign=abi.FFT_NEGATIVE, in_place=True):
        check(load().hpgb_apply_model_fft(self._h, float(norm), int(sign),
                                          1 if in_place else 0))

    def shift_grid(self, direction=abi.SHIFT_FORWARD):
        check(load().hpgb_shift_grid(self._h, int(direction)))

    def shift_model(self, direction=abi.SHIFT_FORWARD):
        check(load().hpgb_shift_model(self._h, int(direction)))

    def set_tiled_plan(self, ring_parts=0, chunk_vis=0, tile_side=0,
                       compensated=0):
        """Override the tiled kernel's plan: ring depth (in largest CF
        parts), visibilities per tile pass, uv tile side (cells) and, in the
        mixed form, compensated tiles (abi.COMPENSATED_ON / _OFF); 0 keeps
        the automatic choice."""
        plan = abi.TiledPlan(int(ring_parts), int(chunk_vis), int(tile_side),
                             int(compensated))
        check(load().hpgb_set_tiled_plan_ex(self._h, ctypes.byref(plan)))

    def tiled_plan(self):
        """The plan overrides in force: dict of ring_parts, chunk_vis,
        tile_side, compensated (0 = automatic)."""
        plan = abi.TiledPlan()
        check(load().hpgb_get_tiled_plan(self._h, ctypes.byref(plan)))
        return {f: getattr(plan, f) for f, _ in abi.TiledPlan._fields_}

    def autotune_tiled(self, visibilities, flags=None, on_device=False):
        """Time the tiled kernel's candidate plans on this batch (grid and
        weights are left unchanged) and keep the fastest; returns
        (ring_parts, chunk_vis)."""
        if flags is None:
            flags = abi.DO_DEGRID | abi.DO_GRID | abi.UPDATE_GRID_WEIGHTS
        ring = ctypes.c_int()
        chunk = ctypes.c_int()
        if on_device:
            n = (visibilities.numel() * visibilities.element_size() //
                 abi.visdata_dtype(self.npol).itemsize)
        else:
            visibilities = np.ascontiguousarray(visibilities)
            n = len(visibilities)
        check(load().hpgb_autotune_tiled(self._h, ptr(visibilities), n,
                                         self.npol, int(flags),
                                         int(bool(on_device)),
                                         ctypes.byref(ring),
                                         ctypes.byref(chunk)))
        return ring.value, chunk.value

    def capture(self):
        """Context manager recording the calls inside it into a CUDA graph
        (see hpgb_begin_capture); yields a Graph filled in at exit."""
        return _Capture(self)

    def profile_tiled_kernel(self, enable=True):
        """Record CUDA events around every tiled-kernel launch (benchmark
        instrumentation)."""
        check(load().hpgb_profile_tiled_kernel(self._h, int(bool(enable))))

    def tiled_kernel_time(self):
        """(summed device ms, launches) of the tiled-kernel launches recorded
        since the last call; waits for the gridder's stream."""
        ms = ctypes.c_double()
        n = ctypes.c_uint64()
        check(load().hpgb_tiled_kernel_time(self._h, ctypes.byref(ms),
                                            ctypes.byref(n)))
        return ms.value, n.value

    def set_wait_limit(self, seconds):
        """Bound of every device-side wait of the tiled kernel (seconds)."""
        check(load().hpgb_set_wait_limit(self._h, float(seconds)))

    def debug_withhold_copy(self, visibility):
        """Test hook: in later tiled launches, the grid-row-0 CTA that takes
        the visibility at this position of the tile-sorted batch never
        issues its copies (-1: none), so that the kernel takes its
        wait-timeout path."""
        check(load().hpgb_debug_withhold_copy(self._h, int(visibility)))

    def last_gridding_kernel(self):
        """abi.KERNEL_TILED or abi.KERNEL_DIRECT: the kernel that took the
        last non-empty batch (abi.KERNEL_AUTO before any)."""
        k = ctypes.c_int()
        check(load().hpgb_last_gridding_kernel(self._h, ctypes.byref(k)))
        return k.value

    def kernel_launches(self):
        """Kernels this gridder has launched so far."""
        n = ctypes.c_uint64()
        check(load().hpgb_kernel_launches(self._h, ctypes.byref(n)))
        return n.value

    def debug_coords(self, visibilities):
        vis = np.ascontiguousarray(visibilities)
        out = np.zeros(len(vis), abi.COORDS_DTYPE)
        check(load().hpgb_debug_coords(self._h, ptr(vis), len(vis), self.npol,
                                       ptr(out)))
        return out


class Graph:
    """An instantiated CUDA graph of a gridder's captured calls."""

    def __init__(self, gridder):
        self._g = gridder
        self._h = None

    def launch(self):
        check(load().hpgb_graph_launch(self._g._h, self._h))

    def close(self):
        if self._h:
            check(load().hpgb_graph_destroy(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _Capture:
    def __init__(self, gridder):
        self.graph = Graph(gridder)

    def __enter__(self):
        check(load().hpgb_begin_capture(self.graph._g._h))
        return self.graph

    def __exit__(self, exc_type, exc, tb):
        h = ctypes.c_void_p()
        rc = load().hpgb_end_capture(self.graph._g._h, ctypes.byref(h))
        if exc_type is None:
            check(rc)
            self.graph._h = h
        elif rc == 0 and h:
            load().hpgb_graph_destroy(h)
        return False


def grid_visibilities_batch(gridders, visibilities, update_grid_weights=True,
                            do_degrid=False, return_visibilities=False,
                            on_device=False):
    """The batches of many gridders in one launch of the tiled kernel
    (hpgb_grid_visibilities_batch): gridders[j] grids visibilities[j] as
    its own grid_visibilities / degrid_grid_visibilities call would.  With
    return_visibilities, returns one Future per gridder (resolved by
    gridders[0].fence()).  Host record arrays, or CUDA uint8 tensors with
    on_device."""
    n = len(gridders)
    if n == 0 or len(visibilities) != n:
        raise ValueError("one batch per gridder")
    npol = gridders[0].npol
    rec = abi.visdata_dtype(npol).itemsize
    flags = abi.DO_GRID | (abi.UPDATE_GRID_WEIGHTS if update_grid_weights else 0)
    if do_degrid:
        flags |= abi.DO_DEGRID
    if return_visibilities:
        flags |= abi.RETURN_VISIBILITIES
    keep, outs = [], []
    hs = (ctypes.c_void_p * n)(*[g._h.value if hasattr(g._h, "value") else g._h
                                 for g in gridders])
    vp = (ctypes.c_void_p * n)()
    nv = (ctypes.c_size_t * n)()
    rp = (ctypes.c_void_p * n)()
    for j, v in enumerate(visibilities):
        if on_device:
            nv[j] = v.numel() * v.element_size() // rec
            vp[j] = v.data_ptr()
            out = v if return_visibilities else None
            if out is not None:
                rp[j] = out.data_ptr()
        else:
            v = np.ascontiguousarray(v)
            keep.append(v)
            nv[j] = len(v)
            vp[j] = v.ctypes.data
            out = np.empty_like(v) if return_visibilities else None
            if out is not None:
                rp[j] = out.ctypes.data
        outs.append(out)
    check(load().hpgb_grid_visibilities_batch(
        hs, n, vp, nv, npol, flags, 1 if on_device else 0, rp))
    if return_visibilities:
        return [Future(gridders[0], o) for o in outs]
    return None
