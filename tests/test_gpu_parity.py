"""Parity of the sm_100a device with the CPU oracle, through the C ABI.

Tolerances (plain FP64 form):
  - coordinates, CF indices, Mueller routing: bit-exact;
  - gridding: grid and weights within 1e-12 relative (the FP32 products are
    computed with the reference's rounding, only FP64 summation order
    differs);
  - degridding: predictions are complex<float>; each within 4 float ulps
    of its magnitude (FP64 sums of different order rounded to float);
  - degrid+grid: at least 99% of the visibilities' residuals must be
    bit-exact (the rest inherit the rare one-ulp differences of the
    prediction); the grid is held to 1e-12 against the oracle's gridding of
    the device's own residuals, and to a norm-wise 1e-6 against the
    oracle's own degrid+grid.
"""
import json
import os

import numpy as np
import pytest

import hpg_b200
from hpg_b200 import Gridder, CFArray, HpgError, workloads
from hpg_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
pytestmark = pytest.mark.gpu


KERNELS = [("direct", abi.PRECISION_FP64), ("tiled", abi.PRECISION_FP64),
           ("tiled", abi.PRECISION_MIXED)]
KERNEL_IDS = ["direct-fp64", "tiled-fp64", "tiled-mixed"]
KIND = {"auto": abi.KERNEL_AUTO, "direct": abi.KERNEL_DIRECT,
        "tiled": abi.KERNEL_TILED}


def make_pair(cfg, oracle_lib, max_batch=None, precision=abi.PRECISION_FP64,
              kernel="auto"):
    O = oracle_lib
    g = Gridder.create(0, 0, max_batch or max(len(cfg["vis"]), 1), None,
                       cfg["grid_size"], cfg["grid_scale"], cfg["mueller"],
                       cfg["conj_mueller"])
    g.set_precision(precision)
    g.set_gridding_kernel(KIND[kernel])
    g.set_convolution_function(CFArray(cfg["oversampling"], cfg["cf_extents"],
                                       cfg["cf_values"]))
    o = O.Oracle(cfg["grid_size"], cfg["grid_scale"], cfg["mueller"],
                 cfg["conj_mueller"], cfg["oversampling"], cfg["cf_extents"],
                 cfg["cf_values"])
    if cfg.get("model") is not None:
        g.set_model(cfg["model"])
        o.set_model(cfg["model"])
    return g, o


def rel_norm(a, b):
    d = np.linalg.norm((a - b).ravel())
    n = np.linalg.norm(b.ravel())
    return d / n if n > 0 else d


def regrid_residuals(cfg, oracle_lib, res):
    """The oracle's gridding of the device's residual visibilities: the
    plain FP64 form's degrid+grid grid must equal it to 1e-12."""
    o = oracle_lib.Oracle(cfg["grid_size"], cfg["grid_scale"], cfg["mueller"],
                          cfg["conj_mueller"], cfg["oversampling"],
                          cfg["cf_extents"], cfg["cf_values"])
    o.grid_visibilities(res)
    return o.grid


def small_full_pol(n=2000, grad=None, seed=7):
    return workloads.full_pol_config(n, grid=256, oversampling=16,
                                     supports=(4, 6, 8, 10), seed=seed,
                                     grad=grad)


def test_coords_bit_exact(gpu, oracle_lib):
    cfg = small_full_pol(5000, grad=0.5)
    rng = np.random.default_rng(3)
    vis = cfg["vis"]
    # half-integer and near-edge positions exercise the rounding branches
    inv_lambda = vis["freq"][0] / 299792458.0
    k = 500
    cells = rng.integers(-100, 100, (k, 2)) + 0.5
    vis["uvw"][:k, 0] = cells[:, 0] / (cfg["grid_scale"][0] * inv_lambda)
    vis["uvw"][:k, 1] = cells[:, 1] / (cfg["grid_scale"][1] * inv_lambda)
    vis["uvw"][k:2 * k, 0] = rng.uniform(-3000, 3000, k)  # partly off grid
    # conjugate Mueller indexes transposed: the routing differs by sign of w
    cfg["conj_mueller"] = [[c * 4 + r for c in range(4)] for r in range(4)]
    g, o = make_pair(cfg, oracle_lib)
    dc = g.debug_coords(vis)
    oc = o.vis_coords(vis)
    for name in oc.dtype.names:
        assert np.array_equal(dc[name], oc[name]), name
    assert (oc["in_grid"] == 0).any() and (oc["in_grid"] == 1).any()
    # Mueller routing: gridding uses the Mueller indexes for w > 0 and the
    # conjugate ones otherwise; degridding the reverse
    pos = dc["pos_w"] == 1
    assert pos.any() and (~pos).any()
    mi, ci = np.array(cfg["mueller"]), np.array(cfg["conj_mueller"])
    assert (dc["grid_mueller"][pos] == mi).all()
    assert (dc["grid_mueller"][~pos] == ci).all()
    assert (dc["degrid_mueller"][pos] == ci).all()
    assert (dc["degrid_mueller"][~pos] == mi).all()


def test_gridone_golden(gpu, oracle_lib):
    """GridderState.GridOne on the device (tests/GridderStateUnitTests.cc
    :1343-1463): footprint exact, values equal to the oracle's and to the
    reference's golden grid where the CF values agree."""
    O = oracle_lib
    golden = np.load(os.path.join(HERE, "golden", "gridone.npy"))
    meta = json.load(open(os.path.join(HERE, "golden", "gridone.json")))
    cf = O.cone_cf(1, meta["cf_oversampling"], meta["cf_radius"])
    cfg = dict(grid_size=meta["grid_size"], grid_scale=meta["grid_scale"],
               mueller=[[0]], conj_mueller=[[0]],
               oversampling=meta["cf_oversampling"], cf_extents=[cf.shape],
               cf_values=[cf])
    g, o = make_pair(cfg, oracle_lib, max_batch=1)
    vd = np.zeros(1, hpg_b200.visdata_dtype(1))
    vd["vis"][0] = complex(*meta["vis"])
    vd["weights"][0] = meta["weight"]
    vd["freq"] = meta["freq"]
    vd["uvw"][0] = meta["uvw"]
    g.grid_visibilities(vd)
    o.grid_visibilities(vd)
    grid = g.grid_values()
    x0, y0 = meta["footprint_ll"]
    sub = grid[0, 0, y0:y0 + 91, x0:x0 + 91].T
    assert np.count_nonzero(grid) == np.count_nonzero(sub)
    assert np.array_equal(grid, o.grid)
    assert np.count_nonzero(sub == golden) >= 8171
    rel = np.abs(sub - golden) / np.maximum(np.abs(golden), 1e-300)
    assert rel[golden != 0].max() <= 2e-7
    w = g.grid_weights()
    assert abs(w[0, 0] - o.weights[0, 0]) <= 1e-12 * abs(o.weights[0, 0])


def test_gridding_sweep(gpu, oracle_lib):
    """GridderState.Gridding (:1273-1341): every fine offset."""
    O = oracle_lib
    cf = O.cone_cf(1, 10, 3)
    cfg = dict(grid_size=(14, 14, 1, 1), grid_scale=(0.1, 0.1), mueller=[[0]],
               conj_mueller=[[0]], oversampling=10, cf_extents=[cf.shape],
               cf_values=[cf])
    for i in range(11):
        for j in range(11):
            g, o = make_pair(cfg, oracle_lib, max_batch=1)
            vd = np.zeros(1, hpg_b200.visdata_dtype(1))
            vd["vis"][0] = 1 - 1j
            vd["weights"][0] = 1.0
            vd["freq"] = 299792458.0
            vd["uvw"][0] = (i * 1.0, j * 1.0, 0.0)
            g.grid_visibilities(vd)
            o.grid_visibilities(vd)
            assert np.array_equal(g.grid_values(), o.grid)
            g.close()


@pytest.mark.parametrize("kernel,precision", KERNELS, ids=KERNEL_IDS)
@pytest.mark.parametrize("npol", [1, 2, 4])
def test_gridding_parity(gpu, oracle_lib, npol, kernel, precision):
    rng = np.random.default_rng(11 + npol)
    gs = (200, 180, npol, 2)
    os_ = 12
    ext, vals = workloads.separable_cf([4, 7, 10], os_,
                                       rng.standard_normal(npol * npol) +
                                       1j * rng.standard_normal(npol * npol),
                                       ncube=2)
    mi = [[r * npol + c for c in range(npol)] for r in range(npol)]
    ci = [[c * npol + r for c in range(npol)] for r in range(npol)]
    vis = workloads.visibilities(3000, npol, gs, (0.05, -0.07), 1.2e9, rng,
                                 w_frac=0.2, ngroups=3, grad=0.4, phase=0.0,
                                 ncube_cf=2)
    vis["phase"] = rng.uniform(-3, 3, len(vis))
    vis["grid_cube"] = rng.integers(0, 2, len(vis))
    cfg = dict(grid_size=gs, grid_scale=(0.05, -0.07), mueller=mi,
               conj_mueller=ci, oversampling=os_, cf_extents=ext,
               cf_values=vals, vis=vis)
    g, o = make_pair(cfg, oracle_lib, precision=precision, kernel=kernel)
    g.grid_visibilities(vis)
    o.grid_visibilities(vis)
    tol = 1e-12 if precision == abi.PRECISION_FP64 else 1e-6
    assert rel_norm(g.grid_values(), o.grid) <= tol
    np.testing.assert_allclose(g.grid_weights(), o.weights, rtol=1e-12)


@pytest.mark.parametrize("kernel,precision", KERNELS, ids=KERNEL_IDS)
def test_degrid_predicted_parity(gpu, oracle_lib, kernel, precision):
    cfg = small_full_pol(3000, grad=0.3)
    g, o = make_pair(cfg, oracle_lib, precision=precision, kernel=kernel)
    fut = g.degrid_get_predicted_visibilities(cfg["vis"])
    assert fut.get() is None
    g.fence()
    got = fut.get()
    exp = o.grid_visibilities(cfg["vis"], update_weights=False, do_degrid=True,
                              return_vis=True, do_grid=False)
    a, b = got["vis"], exp["vis"]
    if precision == abi.PRECISION_FP64:
        ulp = np.spacing(np.maximum(np.abs(b.real),
                                    np.abs(b.imag)).astype(np.float32))
        assert (np.abs(a - b) <= 4 * ulp).all()
        assert np.mean(a == b) > 0.99
    else:
        assert rel_norm(a, b) <= 1e-6


@pytest.mark.parametrize("kernel,precision", KERNELS, ids=KERNEL_IDS)
@pytest.mark.parametrize("grad", [None, 0.4])
def test_degrid_grid_parity(gpu, oracle_lib, grad, kernel, precision):
    cfg = small_full_pol(3000, grad=grad)
    g, o = make_pair(cfg, oracle_lib, precision=precision, kernel=kernel)
    fut = g.degrid_grid_get_residual_visibilities(cfg["vis"])
    g.fence()
    res = fut.get()
    exp = o.grid_visibilities(cfg["vis"], do_degrid=True, return_vis=True)
    grid = g.grid_values()
    if precision == abi.PRECISION_FP64:
        assert np.mean(np.all(res["vis"] == exp["vis"], axis=1)) > 0.99
        assert rel_norm(grid, regrid_residuals(cfg, oracle_lib, res)) <= 1e-12
    else:
        assert rel_norm(res["vis"], exp["vis"]) <= 1e-6
    assert rel_norm(grid, o.grid) <= 1e-6
    np.testing.assert_allclose(g.grid_weights(), o.weights, rtol=1e-12)


@pytest.mark.parametrize("precision,comp",
                         [(abi.PRECISION_FP64, 0), (abi.PRECISION_MIXED, 0),
                          (abi.PRECISION_MIXED, abi.COMPENSATED_ON)],
                         ids=["fp64", "mixed", "mixed-comp"])
@pytest.mark.parametrize("ring_parts,chunk,side",
                         [(4, 64, 0), (6, 0, 0), (5, 7, 0), (4, 1, 0),
                          (5, 2, 0), (3, 0, 0), (2, 5, 0), (4, 0, 20),
                          (5, 3000, 16)])
def test_tiled_plan_overrides(gpu, oracle_lib, precision, comp, ring_parts,
                              chunk, side):
    """Every ring depth, tile side and tile-pass length the plan accepts,
    with and without compensated tiles, gives the same results: small
    chunks cross many tile flushes, a deep ring keeps many visibilities in
    flight, a small side multiplies the tiles."""
    cfg = small_full_pol(3000, grad=0.4)
    g, o = make_pair(cfg, oracle_lib, precision=precision, kernel="tiled")
    g.set_tiled_plan(ring_parts, chunk, side, comp)
    assert g.tiled_plan() == dict(ring_parts=ring_parts, chunk_vis=chunk,
                                  tile_side=side, compensated=comp)
    fut = g.degrid_grid_get_residual_visibilities(cfg["vis"])
    g.fence()
    exp = o.grid_visibilities(cfg["vis"], do_degrid=True, return_vis=True)
    res = fut.get()
    grid = g.grid_values()
    if precision == abi.PRECISION_FP64:
        assert np.mean(np.all(res["vis"] == exp["vis"], axis=1)) > 0.99
        assert rel_norm(grid, regrid_residuals(cfg, oracle_lib, res)) <= 1e-12
    else:
        assert rel_norm(res["vis"], exp["vis"]) <= 1e-6
    assert rel_norm(grid, o.grid) <= 1e-6
    np.testing.assert_allclose(g.grid_weights(), o.weights, rtol=1e-12)


@pytest.mark.parametrize("precision", [abi.PRECISION_FP64, abi.PRECISION_MIXED],
                         ids=["fp64", "mixed"])
def test_autotune_keeps_data_and_parity(gpu, oracle_lib, precision):
    """The autotuner leaves grid and weights as they were and its chosen
    plan gives the same results."""
    cfg = small_full_pol(3000, grad=0.4, seed=9)
    g, o = make_pair(cfg, oracle_lib, precision=precision, kernel="tiled")
    first = cfg["vis"][:1000]
    g.degrid_grid_visibilities(first)
    o.grid_visibilities(first, do_degrid=True)
    g.fence()
    before = (g.grid_values(), g.grid_weights())
    ring, chunk = g.autotune_tiled(cfg["vis"])
    assert 2 <= ring <= 8 and chunk >= 0
    plan = g.tiled_plan()
    assert plan["ring_parts"] == ring and plan["chunk_vis"] == chunk
    # the same workload again: the cached plan, at once
    assert g.autotune_tiled(cfg["vis"]) == (ring, chunk)
    assert np.array_equal(g.grid_values(), before[0])
    assert np.array_equal(g.grid_weights(), before[1])
    rest = cfg["vis"][1000:]
    fut = g.degrid_grid_get_residual_visibilities(rest)
    g.fence()
    exp = o.grid_visibilities(rest, do_degrid=True, return_vis=True)
    if precision == abi.PRECISION_FP64:
        assert np.mean(np.all(fut.get()["vis"] == exp["vis"], axis=1)) > 0.99
    assert rel_norm(g.grid_values(), o.grid) <= 1e-6
    np.testing.assert_allclose(g.grid_weights(), o.weights, rtol=1e-12)


@pytest.mark.parametrize("kernel,precision", KERNELS, ids=KERNEL_IDS)
def test_graph_capture_replay(gpu, oracle_lib, kernel, precision):
    """A degrid+grid call captured into a CUDA graph and replayed three
    times does what three calls do."""
    import torch
    cfg = small_full_pol(2000, grad=0.3, seed=13)
    dv = torch.from_numpy(cfg["vis"].view(np.uint8)).cuda()
    ref, _ = make_pair(cfg, oracle_lib, precision=precision, kernel=kernel)
    for _ in range(3):
        ref.degrid_grid_visibilities(dv, on_device=True)
    ref.fence()
    g, _ = make_pair(cfg, oracle_lib, precision=precision, kernel=kernel)
    g.degrid_grid_visibilities(dv, on_device=True)   # buffers reach size
    g.fence()
    g.reset_grid()
    with g.capture() as graph:
        g.degrid_grid_visibilities(dv, on_device=True)
    before = g.kernel_launches()
    for _ in range(3):
        graph.launch()
    g.fence()
    assert g.kernel_launches() > before
    tol = 1e-12 if precision == abi.PRECISION_FP64 else 1e-6
    assert rel_norm(g.grid_values(), ref.grid_values()) <= tol
    np.testing.assert_allclose(g.grid_weights(), ref.grid_weights(), rtol=1e-12)
    graph.close()
    g.close()
    ref.close()


def test_tiled_plan_rejects_bad_overrides(gpu, oracle_lib):
    """Ring depths outside 2..16 and negative pass lengths are refused."""
    cfg = small_full_pol(10)
    g, _ = make_pair(cfg, oracle_lib, kernel="tiled")
    for bad in ((1, 0), (-1, 0), (17, 0), (0, -1), (0, 0, 129),
                (0, 0, 33), (0, 0, -2), (0, 0, 0, 3)):
        with pytest.raises(HpgError):
            g.set_tiled_plan(*bad)
    g.set_tiled_plan(0, 0)


@pytest.mark.parametrize("kernel,precision", KERNELS, ids=KERNEL_IDS)
def test_degrid_grid_no_model(gpu, oracle_lib, kernel, precision):
    """Without a model the residual is the input (src/hpg_core.hpp:614)."""
    cfg = small_full_pol(2000)
    cfg["model"] = None
    g, o = make_pair(cfg, oracle_lib, precision=precision, kernel=kernel)
    fut = g.degrid_grid_get_residual_visibilities(cfg["vis"])
    g.fence()
    exp = o.grid_visibilities(cfg["vis"], do_degrid=True, return_vis=True)
    assert np.array_equal(fut.get()["vis"], exp["vis"])
    tol = 1e-12 if precision == abi.PRECISION_FP64 else 1e-6
    assert rel_norm(g.grid_values(), o.grid) <= tol


@pytest.mark.parametrize("kernel,precision", KERNELS, ids=KERNEL_IDS)
def test_multi_batch_and_cubes(gpu, oracle_lib, kernel, precision):
    """Several batches into one grid; several grid cubes and CF cubes."""
    rng = np.random.default_rng(21)
    gs = (160, 150, 2, 3)
    ext, vals = workloads.separable_cf([6, 9], 8, [1.0, 0.3 - 0.2j, 0.1j, 0.9],
                                       ncube=2)
    mi = [[0, 1], [2, 3]]
    cfg = dict(grid_size=gs, grid_scale=(0.05, 0.05), mueller=mi,
               conj_mueller=mi, oversampling=8, cf_extents=ext,
               cf_values=vals,
               model=rng.standard_normal((3, 2, 150, 160)) + 0j)
    g, o = make_pair(cfg, oracle_lib, max_batch=2000, precision=precision,
                     kernel=kernel)
    for b in range(3):
        vis = workloads.visibilities(2000, 2, gs, (0.05, 0.05), 1.1e9, rng,
                                     w_frac=0.1, ngroups=2, ncube_cf=2,
                                     grad=0.2)
        vis["grid_cube"] = rng.integers(0, 3, len(vis))
        g.degrid_grid_visibilities(vis)
        o.grid_visibilities(vis, do_degrid=True)
    assert rel_norm(g.grid_values(), o.grid) <= 1e-6
    np.testing.assert_allclose(g.grid_weights(), o.weights, rtol=1e-12)


@pytest.mark.parametrize("precision", [abi.PRECISION_FP64, abi.PRECISION_MIXED],
                         ids=["fp64", "mixed"])
def test_pinned_batches_back_to_back(gpu, oracle_lib, precision):
    """Host batches in pinned memory, four calls without a fence between
    them: each call's copy runs while the previous call's work is on the
    device (two staging buffers in turn); the last call returns residuals."""
    import torch
    cfg = small_full_pol(4000, grad=0.3, seed=17)
    g, o = make_pair(cfg, oracle_lib, max_batch=2000, precision=precision,
                     kernel="tiled")
    halves = [cfg["vis"][:2000], cfg["vis"][2000:]]
    pinned = []
    for h in halves:
        t = torch.from_numpy(np.frombuffer(h.tobytes(), np.uint8).copy()).pin_memory()
        pinned.append(t.numpy().view(h.dtype))
    for k in range(3):
        g.degrid_grid_visibilities(pinned[k % 2])
        o.grid_visibilities(halves[k % 2], do_degrid=True)
    fut = g.degrid_grid_get_residual_visibilities(pinned[1])
    exp = o.grid_visibilities(halves[1], do_degrid=True, return_vis=True)
    g.fence()
    res = fut.get()
    if precision == abi.PRECISION_FP64:
        assert np.mean(np.all(res["vis"] == exp["vis"], axis=1)) > 0.99
    else:
        assert rel_norm(res["vis"], exp["vis"]) <= 1e-6
    assert rel_norm(g.grid_values(), o.grid) <= 1e-6
    np.testing.assert_allclose(g.grid_weights(), o.weights, rtol=1e-12)


def test_cf_device_layouts_match(gpu, oracle_lib):
    """A CF given in the reference's "0-Cuda" or "0-Serial" layout grids
    like the same CF in logical order (DeviceCFArray.Gridding,
    tests/DeviceCFArrayUnitTests.cc:458-547)."""
    cfg = small_full_pol(500)
    os_ = cfg["oversampling"]
    grids = []
    for layout in (None, "0-Cuda", "0-Serial"):
        vals = []
        for ext, v in zip(cfg["cf_extents"], cfg["cf_values"]):
            if layout is None:
                vals.append(v)
                continue
            xm, ym = -(-ext[0] // os_), -(-ext[1] // os_)
            buf = np.zeros((ym * os_, xm * os_, ext[2], ext[3]), np.complex64)
            full = np.zeros((xm * os_, ym * os_, ext[2], ext[3]), np.complex64)
            full[:ext[0], :ext[1]] = v
            # full[x, y, m, c] with x = xmaj*os + xmin
            f = full.reshape(xm, os_, ym, os_, ext[2], ext[3])
            # axes: xmaj, xmin, ymaj, ymin, m, c
            if layout == "0-Cuda":   # Left [xmaj, ymaj, m, c, xmin, ymin]
                buf = np.transpose(f, (3, 1, 5, 4, 2, 0)).copy()
            else:                    # order m, ymaj, xmaj, c, xmin, ymin
                buf = np.transpose(f, (3, 1, 5, 0, 2, 4)).copy()
            vals.append(buf.ravel())
        g = Gridder.create(0, 0, 500, None, cfg["grid_size"], cfg["grid_scale"],
                           cfg["mueller"], cfg["conj_mueller"])
        g.set_convolution_function(CFArray(os_, cfg["cf_extents"], vals, layout))
        g.grid_visibilities(cfg["vis"])
        grids.append(g.grid_values())
    assert np.array_equal(grids[0], grids[1])
    assert np.array_equal(grids[0], grids[2])


def test_normalize_fft_shift(gpu, oracle_lib):
    cfg = small_full_pol(1000)
    g, o = make_pair(cfg, oracle_lib)
    g.grid_visibilities(cfg["vis"])
    o.grid_visibilities(cfg["vis"])
    g.normalize_by_weights(2.0)
    o.normalize_by_weights(2.0)
    assert rel_norm(g.grid_values(), o.grid) <= 1e-12
    g.apply_grid_fft(norm=3.0)
    ref = oracle_lib.fft_grid(o.grid, sign_positive=True) / 3.0
    assert rel_norm(g.grid_values(), ref) <= 1e-12
    g.shift_grid(hpg_b200.SHIFT_FORWARD)
    assert rel_norm(g.grid_values(), np.fft.fftshift(ref, axes=(-2, -1))) <= 1e-12
    g.apply_grid_fft(sign=hpg_b200.FFT_NEGATIVE, in_place=False)
    ref2 = oracle_lib.fft_grid(np.fft.fftshift(ref, axes=(-2, -1)),
                               sign_positive=False)
    assert rel_norm(g.grid_values(), ref2) <= 1e-12


@pytest.mark.parametrize("side", [256, 255])
@pytest.mark.parametrize("sign,direction", [(abi.FFT_POSITIVE, abi.SHIFT_FORWARD),
                                            (abi.FFT_NEGATIVE, abi.SHIFT_BACKWARD)])
def test_image_grid_equals_three_calls(gpu, oracle_lib, side, sign, direction):
    """The fused imaging tail against normalize_by_weights, apply_grid_fft
    and shift_grid called in turn."""
    cfg = workloads.full_pol_config(3000, grid=side, oversampling=16,
                                    supports=(4, 6, 8), seed=17)
    g, _ = make_pair(cfg, oracle_lib, kernel="tiled")
    g.grid_visibilities(cfg["vis"])
    g.fence()
    h = g.copy()
    g.normalize_by_weights(0.5)
    g.apply_grid_fft(3.0, sign)
    g.shift_grid(direction)
    h.image_grid(0.5, 3.0, sign, direction)
    a, b = g.grid_values(), h.grid_values()
    assert np.abs(a).max() > 0
    assert rel_norm(b, a) <= 1e-12
    g.close()
    h.close()


@pytest.mark.parametrize("size", [(20, 20), (19, 19), (18, 19), (19, 18)])
def test_shift_cycle(gpu, oracle_lib, size):
    """GridderState.ShiftCycle (:1860-1926)."""
    rng = np.random.default_rng(1)
    gs = (size[0], size[1], 1, 2)
    g = Gridder.create(0, 0, 1, None, gs, (1, 1), [[0]], [[0]])
    m = rng.standard_normal((2, 1, size[1], size[0])) + 0j
    g.set_model(m)
    g.shift_model(hpg_b200.SHIFT_FORWARD)
    assert np.array_equal(g.model_values(), np.fft.fftshift(m, axes=(-2, -1)))
    g.shift_model(hpg_b200.SHIFT_BACKWARD)
    assert np.array_equal(g.model_values(), m)


def test_one_fft_sign(gpu):
    """GridderState.OneFFT (:1704-1741)."""
    g = Gridder.create(0, 0, 15, None, (2048, 2048, 1, 1), (0.12, -0.34),
                       [[0]], [[0]])
    m = np.zeros((1, 1, 2048, 2048), np.complex128)
    g.set_model(m)
    m = g.model_values()
    m[0, 0, 1108, 1024] = 0.825
    g.set_model(m)
    g.apply_model_fft()
    g.shift_model(hpg_b200.SHIFT_FORWARD)
    assert g.model_values()[0, 0, 10, 1070].imag < 0


def test_model_fft_norm(gpu):
    """GridderState.ModelFFT (:1600-1702)."""
    gs = (64, 64, 4, 3)
    g = Gridder.create(0, 0, 15, None, gs, (0.12, -0.34), [[0]] * 4, [[0]] * 4)
    assert not np.any(g.model_values())
    m = np.zeros((3, 4, 64, 64), np.complex128)
    for r in range(4):
        for c in range(3):
            m[c, r, 32, 32] = (r + 1) * 3 + c
    g.set_model(m)
    g.apply_model_fft()
    m0 = g.model_values()
    assert np.any(m0)
    g.set_model(m)
    g.apply_model_fft(norm=0.001)
    np.testing.assert_allclose(g.model_values(), m0 / 0.001, rtol=1e-12)


def test_residual_and_zero_model(gpu, oracle_lib):
    """ResidualVisibilities (:1743-1815) and ZeroModel (:1523-1598)."""
    O = oracle_lib
    cf = O.cone_cf(1, 10, 3)
    cfg = dict(grid_size=(20, 20, 2, 1), grid_scale=(0.0476591, 0.0476591),
               mueller=[[0, -1], [-1, 0]], conj_mueller=[[0, -1], [-1, 0]],
               oversampling=10, cf_extents=[cf.shape], cf_values=[cf])
    g, _ = make_pair(cfg, oracle_lib, max_batch=1)
    vd = np.zeros(1, hpg_b200.visdata_dtype(2))
    vd["vis"][0] = [1 - 1j, -1 + 1j]
    vd["weights"][0] = [1.0, 0.5]
    vd["freq"] = 3.693e9
    vd["uvw"][0] = (0, 0, 0.1)
    fut = g.degrid_grid_get_residual_visibilities(vd)
    assert fut.get() is None
    g.fence()
    res = fut.get()
    for name in vd.dtype.names:
        assert np.array_equal(res[name], vd[name])
    g1 = g.copy()
    g1.reset_grid()
    g1.grid_visibilities(vd)
    g2 = g.copy()
    g2.reset_grid()
    g2.set_model(np.zeros((1, 2, 20, 20), np.complex128))
    g2.grid_visibilities(vd)
    a, b = g1.grid_values(), g2.grid_values()
    assert np.any(a) and np.array_equal(a, b)


def test_grid_none_and_empty_cf(gpu):
    """GridNone (:1465-1521), EmptyCF (:1817-1858)."""
    empty = CFArray(20, [(31 * 20, 31 * 20, 0, 0)], [np.zeros(0, np.complex64)])
    g = Gridder.create(0, 0, 1, empty, (1024, 1024, 1, 1), (0.05, 0.05),
                       [[0]], [[0]])
    g.grid_visibilities(np.zeros(0, hpg_b200.visdata_dtype(1)))
    assert not np.any(g.grid_values()) and not np.any(g.grid_weights())
    g.set_convolution_function(empty)
    g.grid_visibilities(np.zeros(0, hpg_b200.visdata_dtype(1)))
    assert not np.any(g.grid_values()) and not np.any(g.grid_weights())


def test_errors(gpu, oracle_lib):
    """Error values of the reference (GridderState.ConstructorArgs,
    Batching, GriddingError, CFError: :582-648, :1223-1271, :1085-1124,
    :901-963)."""
    O = oracle_lib
    cf = O.cone_cf(1, 10, 3)
    with pytest.raises(HpgError) as e:
        Gridder.create(0, 0, 1, None, (20, 20, 2, 1), (1, 1), [[0]], [[0]])
    assert e.value.type == "InvalidNumberMuellerIndexRows"
    with pytest.raises(HpgError) as e:
        Gridder.create(99, 0, 1, None, (20, 20, 1, 1), (1, 1), [[0]], [[0]])
    assert e.value.type == "DisabledDevice"
    g = Gridder.create(0, 0, 2, None, (20, 20, 1, 1), (0.05, 0.05), [[0]], [[0]])
    with pytest.raises(HpgError) as e:
        g.set_convolution_function(CFArray(10, [(300, 300, 1, 1)],
                                           [np.zeros((300, 300, 1, 1), np.complex64)]))
    assert e.value.type == "CFSupportExceedsGrid"
    g.set_convolution_function(CFArray(10, [cf.shape], [cf]))
    vd = np.zeros(3, hpg_b200.visdata_dtype(1))
    vd["freq"] = 1e9
    with pytest.raises(HpgError) as e:
        g.grid_visibilities(vd)
    assert e.value.type == "ExcessiveNumberVisibilities"
    with pytest.raises(HpgError) as e:
        g.raw_grid_visibilities(np.zeros(1, hpg_b200.visdata_dtype(2)),
                                abi.DO_GRID, npol=2)
    assert e.value.type == "InvalidNumberPolarizations"
    with pytest.raises(HpgError) as e:
        g.raw_grid_visibilities(vd[:1], abi.UPDATE_GRID_WEIGHTS | abi.DO_DEGRID)
    assert e.value.type == "UpdateWeightsWithoutGridding"
    bad = vd[:1].copy()
    bad["cf_index"][0] = (0, 5)
    with pytest.raises(HpgError) as e:
        g.grid_visibilities(bad)
    assert e.value.type == "OutOfBoundsCFIndex"
    with pytest.raises(HpgError) as e:
        g.set_model(np.zeros((1, 1, 20, 21), np.complex128))
    assert e.value.type == "InvalidModelGridSize"
    with pytest.raises(HpgError) as e:
        g.set_convolution_function(CFArray(10, [cf.shape], [cf], layout="7-Cuda"))
    assert e.value.type == "InvalidCFLayout"


def test_device_resident_input_and_bad_index(gpu, oracle_lib):
    """Visibilities already in device memory; an out-of-range cf_index there
    is skipped on the device and reported at the fence."""
    import torch
    cfg = small_full_pol(1000)
    g, o = make_pair(cfg, oracle_lib)
    dv = torch.from_numpy(cfg["vis"].view(np.uint8)).cuda()
    g.grid_visibilities(dv, on_device=True)
    g.fence()
    o.grid_visibilities(cfg["vis"])
    assert rel_norm(g.grid_values(), o.grid) <= 1e-12
    bad = cfg["vis"][:4].copy()
    bad["cf_index"][2] = (0, 99)
    dv = torch.from_numpy(bad.view(np.uint8)).cuda()
    g.grid_visibilities(dv, on_device=True)
    with pytest.raises(HpgError) as e:
        g.fence()
    assert e.value.type == "OutOfBoundsCFIndex"
    g.fence()  # status cleared
