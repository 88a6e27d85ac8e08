"""hpgb_grid_visibilities_noalloc against hpgb_grid_visibilities.

The allocation-free entry point runs the direct kernels with their
per-visibility scratch in a fixed device array; on the same inputs it must
give what the allocating entry point gives with HPGB_KERNEL_DIRECT:
  - degridding has no atomics, so predicted and residual values are
    bit-identical;
  - the grid and the weights come from FP64 atomic adds in a different
    order: within 1e-12 relative.
Each case makes two calls in a row on one gridder (the grid accumulates, the
scratch array is reused).  This file sorts last so that it also runs after
every other GPU test has used the device.
"""
import ctypes

import numpy as np
import pytest

from hpg_b200 import CFArray, Gridder, HpgError, abi, workloads

pytestmark = pytest.mark.gpu


def _gridder(cfg, max_batch):
    g = Gridder.create(0, 0, max_batch, None, cfg["grid_size"],
                       cfg["grid_scale"], cfg["mueller"], cfg["conj_mueller"])
    g.set_gridding_kernel(abi.KERNEL_DIRECT)
    g.set_convolution_function(CFArray(cfg["oversampling"], cfg["cf_extents"],
                                       cfg["cf_values"]))
    if cfg.get("model") is not None:
        g.set_model(cfg["model"])
    return g


def _noalloc(g, dvis, n, flags):
    abi.check(abi.load().hpgb_grid_visibilities_noalloc(
        g._h, ctypes.c_void_p(dvis.data_ptr()), n, g.npol, flags))


def _rel(a, b):
    return np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300)


@pytest.mark.parametrize("flags", [
    abi.DO_DEGRID | abi.DO_GRID | abi.UPDATE_GRID_WEIGHTS,
    abi.DO_GRID | abi.UPDATE_GRID_WEIGHTS,
    abi.DO_DEGRID,
], ids=["degrid-grid", "grid", "degrid"])
def test_noalloc_matches_allocating_entry_point(gpu, flags):
    import torch
    cfg = workloads.full_pol_config(3000, grid=128, oversampling=16,
                                    supports=(4, 6, 8), seed=11, grad=0.2)
    vis = cfg["vis"]
    n = len(vis)
    raw = np.frombuffer(vis.tobytes(), np.uint8)
    ref = _gridder(cfg, n)
    nal = _gridder(cfg, n)
    try:
        for call in range(2):
            want = ref.raw_grid_visibilities(vis, flags | abi.RETURN_VISIBILITIES)
            ref.fence()
            dvis = torch.from_numpy(raw.copy()).to("cuda:0")
            _noalloc(nal, dvis, n, flags)
            nal.fence()
            got = np.frombuffer(dvis.cpu().numpy().tobytes(),
                                abi.visdata_dtype(4))
            if flags & abi.DO_DEGRID:
                assert np.array_equal(got["vis"].view(np.uint32),
                                      want["vis"].view(np.uint32)), call
            if flags & abi.DO_GRID:
                assert _rel(nal.grid_values(), ref.grid_values()) <= 1e-12, call
                assert _rel(nal.grid_weights(), ref.grid_weights()) <= 1e-12, call
                assert np.abs(ref.grid_values()).max() > 0
    finally:
        ref.close()
        nal.close()


def test_noalloc_leaves_device_memory_unchanged(gpu):
    import torch
    cfg = workloads.full_pol_config(2000, grid=128, oversampling=16,
                                    supports=(4, 6, 8), seed=12)
    n = len(cfg["vis"])
    g = _gridder(cfg, n)
    flags = abi.DO_DEGRID | abi.DO_GRID | abi.UPDATE_GRID_WEIGHTS
    try:
        dvis = torch.from_numpy(
            np.frombuffer(cfg["vis"].tobytes(), np.uint8).copy()).to("cuda:0")
        _noalloc(g, dvis, n, flags)   # first call: module load, address lookup
        g.fence()
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info(0)
        _noalloc(g, dvis, n, flags)
        g.fence()
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info(0)
        assert free1 == free0
    finally:
        g.close()


def test_noalloc_rejects_oversize_batch(gpu):
    import torch
    cfg = workloads.full_pol_config(8, grid=128, oversampling=16,
                                    supports=(4, 6, 8), seed=13)
    n = abi.NOALLOC_MAX_VALUES // 4 + 1
    g = _gridder(cfg, n)
    try:
        rec = abi.visdata_dtype(4).itemsize
        dvis = torch.zeros(n * rec, dtype=torch.uint8, device="cuda:0")
        dvis[: 8 * rec] = torch.from_numpy(
            np.frombuffer(cfg["vis"].tobytes(), np.uint8).copy()).to("cuda:0")
        before = ctypes.c_uint64()
        abi.check(abi.load().hpgb_kernel_launches(g._h, ctypes.byref(before)))
        with pytest.raises(HpgError) as e:
            _noalloc(g, dvis, n, abi.DO_GRID)
        assert e.value.type == "ExcessiveNumberVisibilities"
        after = ctypes.c_uint64()
        abi.check(abi.load().hpgb_kernel_launches(g._h, ctypes.byref(after)))
        assert after.value == before.value
        # degridding alone needs no scratch and is not limited by it
        _noalloc(g, dvis[: 8 * rec], 8, abi.DO_DEGRID)
        g.fence()
    finally:
        g.close()
