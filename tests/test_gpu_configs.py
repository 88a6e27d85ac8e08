"""Device parity with the CPU oracle at the benchmark configurations' shapes.

Two workloads are checked exactly as the benchmark defines them:
  - single polarization: 512x512x1x1, one CF group of support 7 at
    oversampling 20 (Gaussian sigma 1 cell), 100k visibilities, plain
    gridding; every kernel and form;
  - full polarization: 2048x2048x4x1, 8 w-plane CF groups with supports
    8..32 (9..33 taps) at oversampling 128 (the real 10 GB CF table), dense
    4x4 Mueller, complex128 N(0,1) model, degrid+grid of 40k visibilities
    (the benchmark's own seeded generator, a prefix-sized batch); both forms
    through the plan the library picks for the batch, the plan the
    benchmark's autotuner picks at 10M visibilities, and the plan the
    autotuner picks for this batch.

Tolerances:
  - FP64 form, gridding: grid and weights within 1e-12 relative;
  - FP64 form, degrid+grid: residual visibilities are complex<float>; each
    within 4 float ulps and at least 99% bit-exact.  The grid is held to
    1e-12 against the oracle's gridding of the device's own residuals (a
    one-ulp flip of a residual otherwise propagates into the grid), and to
    1e-6 against the oracle's own degrid+grid;
  - mixed form: grid and residuals within 1e-6 relative; weights 1e-12.
"""
import numpy as np
import pytest

from hpg_b200 import CFArray, Gridder, abi, workloads

pytestmark = pytest.mark.gpu

KIND = {"direct": abi.KERNEL_DIRECT, "tiled": abi.KERNEL_TILED}
FORMS = [("direct", abi.PRECISION_FP64), ("tiled", abi.PRECISION_FP64),
         ("tiled", abi.PRECISION_MIXED)]
FORM_IDS = ["direct-fp64", "tiled-fp64", "tiled-mixed"]


def rel_norm(a, b):
    d = np.linalg.norm((np.asarray(a) - np.asarray(b)).ravel())
    n = np.linalg.norm(np.asarray(b).ravel())
    return d / n if n > 0 else d


def check_residuals_fp64(got, exp):
    ulp = np.spacing(np.maximum(np.abs(exp.real),
                                np.abs(exp.imag)).astype(np.float32))
    assert (np.abs(got.real - exp.real) <= 4 * ulp).all()
    assert (np.abs(got.imag - exp.imag) <= 4 * ulp).all()
    assert np.mean(np.all(got == exp, axis=1)) > 0.99


@pytest.mark.parametrize("kernel,precision", FORMS, ids=FORM_IDS)
def test_single_pol_config(gpu, oracle_lib, kernel, precision):
    """The single-polarization benchmark configuration, all 100k
    visibilities, gridding with weights."""
    O = oracle_lib
    cfg = workloads.single_pol_config()
    assert len(cfg["vis"]) == 100_000
    g = Gridder.create(0, 0, len(cfg["vis"]), None, cfg["grid_size"],
                       cfg["grid_scale"], cfg["mueller"], cfg["conj_mueller"])
    g.set_precision(precision)
    g.set_gridding_kernel(KIND[kernel])
    g.set_convolution_function(CFArray(cfg["oversampling"], cfg["cf_extents"],
                                       cfg["cf_values"]))
    o = O.Oracle(cfg["grid_size"], cfg["grid_scale"], cfg["mueller"],
                 cfg["conj_mueller"], cfg["oversampling"], cfg["cf_extents"],
                 cfg["cf_values"])
    g.grid_visibilities(cfg["vis"])
    o.grid_visibilities(cfg["vis"], nthreads=O.num_threads())
    grid, wgt = g.grid_values(), g.grid_weights()
    assert np.count_nonzero(o.grid) > 100_000
    tol = 1e-12 if precision == abi.PRECISION_FP64 else 1e-6
    assert rel_norm(grid, o.grid) <= tol
    np.testing.assert_allclose(wgt, o.weights, rtol=1e-12)
    g.close()


# --------------------------------------------------------------------------
# full polarization at the benchmark's shapes

FULL_POL_NVIS = 40_000
# the plans the benchmark's autotuner chose for 10M visibilities of this
# workload (ring parts, visibilities per tile pass)
BENCH_PLANS = {abi.PRECISION_MIXED: (5, 512), abi.PRECISION_FP64: (5, 4096),
               "mixed-comp": (4, 2048)}


@pytest.fixture(scope="module")
def full_pol(gpu, oracle_lib):
    import torch
    O = oracle_lib
    p = workloads.full_pol_params()
    grid_size = (2048, 2048, 4, 1)
    vis = workloads.visibilities(FULL_POL_NVIS, 4, grid_size, p["grid_scale"],
                                 p["freq"], p["rng"], w_frac=0.3,
                                 ngroups=len(p["supports"]))
    dev = torch.device("cuda", 0)
    ext, dvals = workloads.separable_cf_torch(p["supports"], p["oversampling"],
                                              p["mueller_factors"], dev,
                                              w_phases=p["w_phases"])
    hvals = [v.cpu().numpy() for v in dvals]
    model = (p["rng"].standard_normal((1, 4) + grid_size[1::-1]) +
             1j * p["rng"].standard_normal((1, 4) + grid_size[1::-1]))
    o = O.Oracle(grid_size, p["grid_scale"], p["mueller"], p["conj_mueller"],
                 p["oversampling"], ext, hvals)
    o.set_model(model)
    exp_res = o.grid_visibilities(vis, do_degrid=True, return_vis=True,
                                  nthreads=O.num_threads())
    case = dict(p=p, grid_size=grid_size, vis=vis, ext=ext, dvals=dvals,
                hvals=hvals, model=model, exp_res=exp_res, exp_grid=o.grid,
                exp_weights=o.weights)
    yield case
    case.clear()
    torch.cuda.empty_cache()


def _full_pol_gridder(case, kernel, precision):
    p = case["p"]
    g = Gridder.create(0, 0, len(case["vis"]), None, case["grid_size"],
                       p["grid_scale"], p["mueller"], p["conj_mueller"])
    g.set_precision(precision)
    g.set_gridding_kernel(KIND[kernel])
    g.set_convolution_function(CFArray(p["oversampling"], case["ext"],
                                       case["dvals"]), on_device=True)
    g.set_model(case["model"])
    return g


def _check_full_pol(case, oracle_lib, g, precision, res):
    O = oracle_lib
    grid, wgt = g.grid_values(), g.grid_weights()
    np.testing.assert_allclose(wgt, case["exp_weights"], rtol=1e-12)
    if precision == abi.PRECISION_FP64:
        check_residuals_fp64(res["vis"], case["exp_res"]["vis"])
        # the gridding half at the plain form's tolerance: the oracle grids
        # the device's own residuals
        p = case["p"]
        o2 = O.Oracle(case["grid_size"], p["grid_scale"], p["mueller"],
                      p["conj_mueller"], p["oversampling"], case["ext"],
                      case["hvals"])
        o2.grid_visibilities(res, nthreads=O.num_threads())
        assert rel_norm(grid, o2.grid) <= 1e-12
        np.testing.assert_allclose(wgt, o2.weights, rtol=1e-12)
        assert rel_norm(grid, case["exp_grid"]) <= 1e-6
    else:
        assert rel_norm(res["vis"], case["exp_res"]["vis"]) <= 1e-6
        assert rel_norm(grid, case["exp_grid"]) <= 1e-6


@pytest.mark.parametrize("plan", ["default", "bench", "autotuned"])
@pytest.mark.parametrize("precision,comp",
                         [(abi.PRECISION_FP64, 0), (abi.PRECISION_MIXED, 0),
                          (abi.PRECISION_MIXED, abi.COMPENSATED_ON)],
                         ids=["fp64", "mixed", "mixed-comp"])
def test_full_pol_config_tiled(gpu, oracle_lib, full_pol, precision, comp,
                               plan):
    """degrid_grid_get_residual_visibilities at the full-polarization
    benchmark's shapes through the tiled kernel."""
    case = full_pol
    g = _full_pol_gridder(case, "tiled", precision)
    g.set_tiled_plan(compensated=comp)
    if plan == "bench":
        ring, chunk = BENCH_PLANS[precision]
        if comp:
            ring, chunk = BENCH_PLANS["mixed-comp"]
        g.set_tiled_plan(ring, chunk, compensated=comp)
    elif plan == "autotuned":
        ring, chunk = g.autotune_tiled(case["vis"])
        assert 2 <= ring <= 8
        assert g.tiled_plan()["compensated"] == comp
    fut = g.degrid_grid_get_residual_visibilities(case["vis"])
    g.fence()
    _check_full_pol(case, oracle_lib, g, precision, fut.get())
    g.close()


def test_compensated_tiles_error(gpu, oracle_lib, full_pol):
    """Compensated (two-sum) FP32 tiles against plain FP32 tiles at long
    tile passes (8192 visibilities): each mixed-form grid is compared with
    the oracle's gridding of that run's own residuals, which removes the
    degridding error and leaves the gridding products and the tile
    accumulation.  The compensated tiles accumulate without FP32 error, so
    their grid error is at most half the plain tiles' and within 1e-7."""
    O = oracle_lib
    case = full_pol
    p = case["p"]
    # visibilities packed into a disk of 20 cells around the grid centre:
    # thousands share each uv tile, so a tile pass sums thousands of them
    vis = workloads.visibilities(30_000, 4, case["grid_size"],
                                 p["grid_scale"], p["freq"],
                                 np.random.default_rng(77), disk=0.01,
                                 w_frac=0.3, ngroups=len(p["supports"]))
    errs = {}
    for comp in (abi.COMPENSATED_OFF, abi.COMPENSATED_ON):
        g = _full_pol_gridder(case, "tiled", abi.PRECISION_MIXED)
        # four ring parts: the compensated form's four tiles (two groups)
        # leave no room beside five
        g.set_tiled_plan(4, 8192, compensated=comp)
        fut = g.degrid_grid_get_residual_visibilities(vis)
        g.fence()
        o = O.Oracle(case["grid_size"], p["grid_scale"], p["mueller"],
                     p["conj_mueller"], p["oversampling"], case["ext"],
                     case["hvals"])
        o.grid_visibilities(fut.get(), nthreads=O.num_threads())
        errs[comp] = rel_norm(g.grid_values(), o.grid)
        g.close()
    assert errs[abi.COMPENSATED_ON] <= 1e-7
    assert errs[abi.COMPENSATED_ON] <= 0.5 * errs[abi.COMPENSATED_OFF]


def test_full_pol_config_direct(gpu, oracle_lib, full_pol):
    """The same call through the per-visibility kernels (FP64)."""
    case = full_pol
    g = _full_pol_gridder(case, "direct", abi.PRECISION_FP64)
    fut = g.degrid_grid_get_residual_visibilities(case["vis"])
    g.fence()
    _check_full_pol(case, oracle_lib, g, abi.PRECISION_FP64, fut.get())
    g.close()


# --------------------------------------------------------------------------
# wide supports through the tiled kernel

@pytest.mark.parametrize("npol", [1, 2, 4])
@pytest.mark.parametrize("precision", [abi.PRECISION_FP64, abi.PRECISION_MIXED],
                         ids=["fp64", "mixed"])
def test_wide_supports_tiled(gpu, oracle_lib, precision, npol):
    """CF groups of supports 8, 16, 32 and 64 (9..65 taps), diagonal
    Mueller (one plane per grid row), as in the batched and the
    differentiable configurations: the tiled kernel takes the batch (its
    ring holds two or three of the 33 KB parts) and degrid+grid matches the
    oracle."""
    O = oracle_lib
    rng = np.random.default_rng(40 + npol)
    gs = (384, 384, npol, 1)
    supports = (8, 16, 32, 64)
    os_ = 8
    ext, vals = workloads.separable_cf(supports, os_, np.ones(npol) +
                                       0.1j * rng.standard_normal(npol))
    mi = [[r if c == r else -1 for c in range(npol)] for r in range(npol)]
    vis = workloads.visibilities(3000, npol, gs, (0.05, 0.05), 1.4e9, rng,
                                 disk=0.3, w_frac=0.3, ngroups=len(supports),
                                 grad=0.2)
    model = (rng.standard_normal((1, npol, 384, 384)) +
             1j * rng.standard_normal((1, npol, 384, 384)))
    cfg = dict(grid_size=gs, grid_scale=(0.05, 0.05), mueller=mi,
               conj_mueller=mi, oversampling=os_, cf_extents=ext,
               cf_values=vals, vis=vis, model=model)
    g = Gridder.create(0, 0, len(vis), None, gs, cfg["grid_scale"], mi, mi)
    g.set_precision(precision)
    g.set_gridding_kernel(abi.KERNEL_TILED)
    g.set_convolution_function(CFArray(os_, ext, vals))
    g.set_model(model)
    o = O.Oracle(gs, cfg["grid_scale"], mi, mi, os_, ext, vals)
    o.set_model(model)
    fut = g.degrid_grid_get_residual_visibilities(vis)
    g.fence()
    assert g.last_gridding_kernel() == abi.KERNEL_TILED
    res = fut.get()
    exp = o.grid_visibilities(vis, do_degrid=True, return_vis=True)
    grid = g.grid_values()
    # every support class is present
    assert set(np.unique(vis["cf_index"][:, 1])) == {0, 1, 2, 3}
    if precision == abi.PRECISION_FP64:
        check_residuals_fp64(res["vis"], exp["vis"])
        o2 = O.Oracle(gs, cfg["grid_scale"], mi, mi, os_, ext, vals)
        o2.grid_visibilities(res)
        assert rel_norm(grid, o2.grid) <= 1e-12
    else:
        assert rel_norm(res["vis"], exp["vis"]) <= 1e-6
    assert rel_norm(grid, o.grid) <= 1e-6
    np.testing.assert_allclose(g.grid_weights(), o.weights, rtol=1e-12)
    g.close()


def test_fallback_is_reported(gpu, oracle_lib):
    """A dense 4x4 Mueller CF of support 64 does not fit the tiled kernel's
    shared memory (a row's four 33 KB planes): the automatic choice grids it
    with the per-visibility kernels and says so; forcing the tiled kernel
    is an error."""
    from hpg_b200 import HpgError
    rng = np.random.default_rng(3)
    gs = (256, 256, 4, 1)
    mf, idx = workloads.dense_mueller(rng)
    ext, vals = workloads.separable_cf([64], 4, mf)
    vis = workloads.visibilities(200, 4, gs, (0.05, 0.05), 1.4e9, rng,
                                 disk=0.2)
    g = Gridder.create(0, 0, len(vis), None, gs, (0.05, 0.05), idx, idx)
    assert g.last_gridding_kernel() == abi.KERNEL_AUTO
    g.set_convolution_function(CFArray(4, ext, vals))
    g.grid_visibilities(vis)
    g.fence()
    assert g.last_gridding_kernel() == abi.KERNEL_DIRECT
    g.set_gridding_kernel(abi.KERNEL_TILED)
    with pytest.raises(HpgError):
        g.grid_visibilities(vis)
    g.close()


# --------------------------------------------------------------------------
# gridding without weight updates (VisibilityGridder::grid_vis_no_weights,
# src/hpg_core.hpp:994-1068, launched at :1220-1251)

def _small_case(seed=31):
    return workloads.full_pol_config(3000, grid=256, oversampling=16,
                                     supports=(4, 6, 8, 10), seed=seed,
                                     grad=0.3)


@pytest.mark.parametrize("degrid", [False, True], ids=["grid", "degrid+grid"])
@pytest.mark.parametrize("kernel,precision", FORMS, ids=FORM_IDS)
def test_no_weight_update(gpu, oracle_lib, kernel, precision, degrid):
    """update_grid_weights=False leaves the weights at zero and grids what
    the weighted call grids."""
    O = oracle_lib
    cfg = _small_case()
    grids, weights = [], []
    for update in (True, False):
        g = Gridder.create(0, 0, len(cfg["vis"]), None, cfg["grid_size"],
                           cfg["grid_scale"], cfg["mueller"],
                           cfg["conj_mueller"])
        g.set_precision(precision)
        g.set_gridding_kernel(KIND[kernel])
        g.set_convolution_function(CFArray(cfg["oversampling"],
                                           cfg["cf_extents"],
                                           cfg["cf_values"]))
        g.set_model(cfg["model"])
        if degrid:
            g.degrid_grid_visibilities(cfg["vis"], update_grid_weights=update)
        else:
            g.grid_visibilities(cfg["vis"], update_grid_weights=update)
        grids.append(g.grid_values())
        weights.append(g.grid_weights())
        g.close()
    o = O.Oracle(cfg["grid_size"], cfg["grid_scale"], cfg["mueller"],
                 cfg["conj_mueller"], cfg["oversampling"], cfg["cf_extents"],
                 cfg["cf_values"])
    o.set_model(cfg["model"])
    o.grid_visibilities(cfg["vis"], update_weights=False, do_degrid=degrid)
    assert not np.any(o.weights)
    assert not np.any(weights[1])
    assert np.any(weights[0])
    tol = 1e-12 if precision == abi.PRECISION_FP64 else 1e-6
    assert rel_norm(grids[1], grids[0]) <= tol
    assert rel_norm(grids[1], o.grid) <= (1e-6 if degrid else tol)


# --------------------------------------------------------------------------
# reference state tests restated on the device

def _cone_cfg(oracle_lib, seed, nvis, sizes=((3, 3), (2, 2))):
    """GridderStateUnitTests.cc-style state: 16x15x1x3 grid, scale
    (0.1, -0.1), oversampling 10, CF groups of the given (radius, cubes)."""
    rng = np.random.default_rng(seed)
    gs = (16, 15, 1, 3)
    ext, vals = [], []
    for radius, cubes in sizes:
        w = 2 * (radius + 2) * 10 + 1
        v = (rng.uniform(-1, 1, (w, w, 1, cubes)) +
             1j * rng.uniform(-1, 1, (w, w, 1, cubes))).astype(np.complex64)
        ext.append(v.shape)
        vals.append(v)
    vis = np.zeros(nvis, abi.visdata_dtype(1))
    vis["vis"][:, 0] = (rng.uniform(-1, 1, nvis) +
                        1j * rng.uniform(-1, 1, nvis))
    vis["weights"] = rng.uniform(0.5, 1.5, (nvis, 1))
    vis["freq"] = 3.693e9
    inv_lambda = 3.693e9 / 299792458.0
    # footprints inside the grid: positions within +-2 cells of the centre
    vis["uvw"][:, 0] = rng.uniform(-2, 2, nvis) / (0.1 * inv_lambda)
    vis["uvw"][:, 1] = rng.uniform(-2, 2, nvis) / (-0.1 * inv_lambda)
    vis["uvw"][:, 2] = rng.uniform(-1, 1, nvis)
    vis["grid_cube"] = rng.integers(0, 3, nvis)
    return dict(grid_size=gs, grid_scale=(0.1, -0.1), mueller=[[0]],
                conj_mueller=[[0]], oversampling=10, cf_extents=ext,
                cf_values=vals, vis=vis, rng=rng)


def _state(cfg, nvis, precision=abi.PRECISION_FP64, kernel="tiled"):
    g = Gridder.create(0, 0, nvis, None, cfg["grid_size"], cfg["grid_scale"],
                       cfg["mueller"], cfg["conj_mueller"])
    g.set_precision(precision)
    g.set_gridding_kernel(KIND[kernel])
    return g


def _vis_for(cfg, grp_cubes, n, seed):
    """n records of cfg's visibilities re-indexed into a CF of groups with
    grp_cubes[g] cubes."""
    rng = np.random.default_rng(seed)
    v = cfg["vis"][:n].copy()
    grp = rng.integers(0, len(grp_cubes), n)
    v["cf_index"][:, 1] = grp
    v["cf_index"][:, 0] = [rng.integers(0, grp_cubes[k]) for k in grp]
    return v


@pytest.mark.parametrize("kernel,precision", FORMS, ids=FORM_IDS)
def test_serialization(gpu, oracle_lib, kernel, precision):
    """GridderState.Serialization (tests/GridderStateUnitTests.cc:1126-1221):
    two CF sets, each with its own visibilities, gridded in both orders give
    the same grid and weights; run twice, so that the second run reuses the
    CF region.  The reference holds the results to 1e-3; FP64 here to
    1e-12."""
    cfg = _cone_cfg(oracle_lib, 42, 1000)
    cfs = [CFArray(10, [cfg["cf_extents"][0]], [cfg["cf_values"][0]]),
           CFArray(10, [cfg["cf_extents"][1]], [cfg["cf_values"][1]])]
    vis = [_vis_for(cfg, [3], 1000, 1), _vis_for(cfg, [2], 1000, 2)]

    def run(first, second, g):
        g.reset_grid()
        g.set_convolution_function(cfs[first])
        g.grid_visibilities(vis[first])
        g.set_convolution_function(cfs[second])
        g.grid_visibilities(vis[second])
        return g.grid_values(), g.grid_weights()

    tol = 1e-12 if precision == abi.PRECISION_FP64 else 1e-6
    g01 = _state(cfg, 1000, precision, kernel)
    g10 = _state(cfg, 1000, precision, kernel)
    for _ in range(2):
        v01, w01 = run(0, 1, g01)
        v10, w10 = run(1, 0, g10)
        assert np.any(v01)
        assert rel_norm(v10, v01) <= tol
        np.testing.assert_allclose(w10, w01, rtol=1e-12)


@pytest.mark.parametrize("kernel,precision", FORMS, ids=FORM_IDS)
def test_visibility_order_invariance(gpu, oracle_lib, kernel, precision):
    """The tiled path sorts visibilities by tile: any batch order grids the
    same (reversed and shuffled batches against the given order)."""
    cfg = workloads.full_pol_config(4000, grid=256, oversampling=16,
                                    supports=(4, 6, 8, 10), seed=3, grad=0.2)
    rng = np.random.default_rng(5)
    orders = [np.arange(4000), np.arange(4000)[::-1], rng.permutation(4000)]
    out = []
    for order in orders:
        g = _state(cfg, 4000, precision, kernel)
        g.set_convolution_function(CFArray(cfg["oversampling"],
                                           cfg["cf_extents"],
                                           cfg["cf_values"]))
        g.set_model(cfg["model"])
        fut = g.degrid_grid_get_residual_visibilities(cfg["vis"][order])
        g.fence()
        res = fut.get()
        back = np.empty_like(res)
        back[order] = res
        out.append((g.grid_values(), g.grid_weights(), back))
        g.close()
    tol = 1e-12 if precision == abi.PRECISION_FP64 else 1e-6
    for grid, wgt, res in out[1:]:
        assert rel_norm(grid, out[0][0]) <= tol
        np.testing.assert_allclose(wgt, out[0][1], rtol=1e-12)
        # each residual depends on its own visibility only: bit-identical in
        # the FP64 form
        if precision == abi.PRECISION_FP64:
            assert np.array_equal(res["vis"], out[0][2]["vis"])
        else:
            assert rel_norm(res["vis"], out[0][2]["vis"]) <= 1e-6


@pytest.mark.parametrize("kernel,precision", FORMS, ids=FORM_IDS)
def test_sequences(gpu, oracle_lib, kernel, precision):
    """GridderState.Sequences (:1023-1083): gridding calls interleaved with
    set_convolution_function calls, each call's contribution as the
    oracle's."""
    O = oracle_lib
    cfg = _cone_cfg(oracle_lib, 42, 10)
    cf = CFArray(10, cfg["cf_extents"], cfg["cf_values"])
    vis = _vis_for(cfg, [3, 2], 10, 7)
    g = _state(cfg, 10, precision, kernel)
    o = O.Oracle(cfg["grid_size"], cfg["grid_scale"], cfg["mueller"],
                 cfg["conj_mueller"], 10, cfg["cf_extents"], cfg["cf_values"])
    g.set_convolution_function(cf)
    g.grid_visibilities(vis)
    g.grid_visibilities(vis)
    g.set_convolution_function(cf)
    g.grid_visibilities(vis)
    g.grid_visibilities(vis)
    for _ in range(4):
        o.grid_visibilities(vis)
    tol = 1e-12 if precision == abi.PRECISION_FP64 else 1e-6
    assert np.any(o.grid)
    assert rel_norm(g.grid_values(), o.grid) <= tol
    np.testing.assert_allclose(g.grid_weights(), o.weights, rtol=1e-12)


def test_copies_and_reset_with_data(gpu, oracle_lib):
    """GridderState.Copies (:650-687) and Reset (:965-1021) with gridded
    data: a copy keeps the parameters and the data of its source and grids
    on independently; reset_grid of a copy zeroes the copy only."""
    cfg = _cone_cfg(oracle_lib, 42, 10)
    cf = CFArray(10, cfg["cf_extents"], cfg["cf_values"])
    vis = _vis_for(cfg, [3, 2], 10, 9)
    g = _state(cfg, 10)
    g.set_convolution_function(cf)
    g.grid_visibilities(vis)
    values, weights = g.grid_values(), g.grid_weights()
    assert np.any(values) and np.any(weights)
    h = g.copy()
    assert h.grid_size == g.grid_size and h.num_polarizations() == 1
    assert (h.convolution_function_region_size(None) ==
            g.convolution_function_region_size(None) > 0)
    assert np.array_equal(h.grid_values(), values)
    assert np.array_equal(h.grid_weights(), weights)
    h.reset_grid()
    assert not np.any(h.grid_values()) and not np.any(h.grid_weights())
    assert np.array_equal(g.grid_values(), values)
    assert np.array_equal(g.grid_weights(), weights)
    # the copy kept the CF: gridding the batch again reproduces the data
    h.grid_visibilities(vis)
    assert rel_norm(h.grid_values(), values) <= 1e-12
    np.testing.assert_allclose(h.grid_weights(), weights, rtol=1e-12)
    g.grid_visibilities(vis)
    assert rel_norm(g.grid_values(), 2 * values) <= 1e-12
    h.close()
    g.close()
