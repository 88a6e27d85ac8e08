"""One launch of the tiled kernel over the batches of many gridders
(hpgb_grid_visibilities_batch), against the oracle per gridder.

The jobs are uneven on purpose: grid sides 96..400 (some rectangular, one
with two cubes), one to four CF groups with supports 4..16 (and 24 for
some, so that the batch spans two support classes, which take a launch
each on forked streams) at oversampling 8, batches of 0..5000
visibilities, two polarizations with a diagonal Mueller matrix; a second
set reaches support 64 (three support classes).  Gridders of a batch are
split into launches by support class and by their own plan's tile side.  Tolerances as in the single-gridder parity tests:
FP64 gridding 1e-12; mixed 1e-6; FP64 degrid+grid residuals at least 99%
bit-exact, and the grid within 1e-12 of the oracle's gridding of the
device's residuals.
"""
import numpy as np
import pytest

import hpg_b200
from hpg_b200 import CFArray, Gridder, HpgError, abi, workloads

pytestmark = pytest.mark.gpu

MI = [[0, -1], [-1, 1]]
FORMS = [(abi.PRECISION_FP64, 0), (abi.PRECISION_MIXED, 0),
         (abi.PRECISION_MIXED, abi.COMPENSATED_ON)]
FORM_IDS = ["fp64", "mixed", "mixed-comp"]


def rel_norm(a, b):
    return np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel())


def make_jobs(seed=1, njobs=9):
    rng = np.random.default_rng(seed)
    jobs = []
    for j in range(njobs):
        # even widths: the mixed form's FP32 model rows must start on
        # 16-byte boundaries for the tensor copy
        nx = int(rng.integers(48, 200)) * 2
        ny = nx if j % 3 else int(rng.integers(96, 400))
        cubes = 2 if j == 4 else 1
        gs = (nx, ny, 2, cubes)
        ngroups = int(rng.integers(1, 4))
        supports = [int(s) for s in rng.integers(4, 17, ngroups)]
        if j % 4 == 1:  # a wider CF: a second support class, own launch
            supports.append(24)
            ngroups += 1
        ext, vals = workloads.separable_cf(
            supports, 8, np.ones(2) + 0.2j * rng.standard_normal(2))
        n = 0 if j == 7 else int(rng.integers(100, 5000))
        vis = workloads.visibilities(n, 2, gs, (0.05, 0.05), 1.4e9, rng,
                                     disk=0.4 * min(nx, ny) / max(nx, ny),
                                     w_frac=0.2, ngroups=ngroups, grad=0.2)
        if cubes > 1:
            vis["grid_cube"] = rng.integers(0, cubes, n)
        model = (rng.standard_normal((cubes, 2, ny, nx)) +
                 1j * rng.standard_normal((cubes, 2, ny, nx)))
        jobs.append(dict(grid_size=gs, cf_extents=ext, cf_values=vals,
                         vis=vis, model=model))
    return jobs


def gridders_for(jobs, precision, comp, model):
    gs = []
    for job in jobs:
        g = Gridder.create(0, 0, max(len(job["vis"]), 1), None,
                           job["grid_size"], (0.05, 0.05), MI, MI)
        g.set_precision(precision)
        g.set_tiled_plan(compensated=comp)
        g.set_convolution_function(CFArray(8, job["cf_extents"],
                                           job["cf_values"]))
        if model:
            g.set_model(job["model"])
        gs.append(g)
    return gs


def oracle_for(O, job, model):
    o = O.Oracle(job["grid_size"], (0.05, 0.05), MI, MI, 8, job["cf_extents"],
                 job["cf_values"])
    if model:
        o.set_model(job["model"])
    return o


@pytest.mark.parametrize("degrid", [False, True], ids=["grid", "degrid+grid"])
@pytest.mark.parametrize("precision,comp", FORMS, ids=FORM_IDS)
def test_batch_matches_oracle(gpu, oracle_lib, precision, comp, degrid):
    O = oracle_lib
    jobs = make_jobs()
    gs = gridders_for(jobs, precision, comp, degrid)
    futs = hpg_b200.grid_visibilities_batch(
        gs, [j["vis"] for j in jobs], do_degrid=degrid,
        return_visibilities=True)
    gs[0].fence()
    for k, (job, g, fut) in enumerate(zip(jobs, gs, futs)):
        o = oracle_for(O, job, degrid)
        exp = o.grid_visibilities(job["vis"], do_degrid=degrid,
                                  return_vis=True)
        grid, wgt = g.grid_values(), g.grid_weights()
        if len(job["vis"]) == 0:
            assert not np.any(grid) and not np.any(wgt)
            continue
        assert g.last_gridding_kernel() == abi.KERNEL_TILED
        np.testing.assert_allclose(wgt, o.weights, rtol=1e-12)
        res = fut.get()
        if precision == abi.PRECISION_FP64:
            if degrid:
                assert np.mean(np.all(res["vis"] == exp["vis"], axis=1)) > 0.99
                o2 = oracle_for(O, job, False)
                o2.grid_visibilities(res)
                assert rel_norm(grid, o2.grid) <= 1e-12, k
                assert rel_norm(grid, o.grid) <= 1e-6, k
            else:
                assert np.array_equal(res, job["vis"])
                assert rel_norm(grid, o.grid) <= 1e-12, k
        else:
            if degrid:
                assert rel_norm(res["vis"], exp["vis"]) <= 1e-6
            assert rel_norm(grid, o.grid) <= 1e-6, k
    for g in gs:
        g.close()


def make_wide_jobs(seed=5):
    """Gridders whose widest CFs reach support 64 (65 taps: the launch of
    that support class takes a two- or three-part CF ring) beside ones
    whose widest are 32 and 16 (three support classes, a launch or more
    each),
    two polarizations, diagonal Mueller."""
    rng = np.random.default_rng(seed)
    jobs = []
    for supports in ([64], [8, 64], [32], [16, 32], [64, 32, 8], [8, 16]):
        nx = int(rng.integers(80, 160)) * 2
        gs = (nx, nx, 2, 1)
        ext, vals = workloads.separable_cf(
            supports, 8, np.ones(2) + 0.2j * rng.standard_normal(2))
        n = int(rng.integers(300, 1500))
        vis = workloads.visibilities(n, 2, gs, (0.05, 0.05), 1.4e9, rng,
                                     disk=0.3, w_frac=0.2,
                                     ngroups=len(supports), grad=0.2)
        model = (rng.standard_normal((1, 2, nx, nx)) +
                 1j * rng.standard_normal((1, 2, nx, nx)))
        jobs.append(dict(grid_size=gs, cf_extents=ext, cf_values=vals,
                         vis=vis, model=model))
    return jobs


@pytest.mark.parametrize("precision", [abi.PRECISION_FP64, abi.PRECISION_MIXED],
                         ids=["fp64", "mixed"])
def test_batch_wide_supports(gpu, oracle_lib, precision):
    """The batched launches at supports up to 64 (three support classes:
    shallow rings and large tiles for the widest) against the oracle per
    gridder, degrid+grid."""
    O = oracle_lib
    jobs = make_wide_jobs()
    gs = gridders_for(jobs, precision, 0, True)
    futs = hpg_b200.grid_visibilities_batch(
        gs, [j["vis"] for j in jobs], do_degrid=True,
        return_visibilities=True)
    gs[0].fence()
    for k, (job, g, fut) in enumerate(zip(jobs, gs, futs)):
        o = oracle_for(O, job, True)
        exp = o.grid_visibilities(job["vis"], do_degrid=True, return_vis=True)
        assert g.last_gridding_kernel() == abi.KERNEL_TILED
        np.testing.assert_allclose(g.grid_weights(), o.weights, rtol=1e-12)
        res = fut.get()
        grid = g.grid_values()
        if precision == abi.PRECISION_FP64:
            assert np.mean(np.all(res["vis"] == exp["vis"], axis=1)) > 0.99, k
            o2 = oracle_for(O, job, False)
            o2.grid_visibilities(res)
            assert rel_norm(grid, o2.grid) <= 1e-12, k
        else:
            assert rel_norm(res["vis"], exp["vis"]) <= 1e-6, k
        assert rel_norm(grid, o.grid) <= 1e-6, k
    for g in gs:
        g.close()


def test_batch_equals_single_calls(gpu):
    """The batched launch against one call per gridder (FP64, degrid+grid):
    residuals bit-identical, grids within 1e-12 (atomic order)."""
    jobs = make_jobs(seed=2, njobs=6)
    single = gridders_for(jobs, abi.PRECISION_FP64, 0, True)
    batched = gridders_for(jobs, abi.PRECISION_FP64, 0, True)
    res1 = []
    for g, job in zip(single, jobs):
        fut = g.degrid_grid_get_residual_visibilities(job["vis"])
        g.fence()
        res1.append(fut.get())
    futs = hpg_b200.grid_visibilities_batch(
        batched, [j["vis"] for j in jobs], do_degrid=True,
        return_visibilities=True)
    batched[0].fence()
    for a, b, r1, f in zip(single, batched, res1, futs):
        if r1 is not None and len(r1):
            assert np.array_equal(f.get()["vis"], r1["vis"])
            assert rel_norm(b.grid_values(), a.grid_values()) <= 1e-12
        np.testing.assert_allclose(b.grid_weights(), a.grid_weights(),
                                   rtol=1e-12)
    for g in single + batched:
        g.close()


@pytest.mark.parametrize("precision", [abi.PRECISION_FP64, abi.PRECISION_MIXED],
                         ids=["fp64", "mixed"])
def test_batch_graph_capture(gpu, precision):
    """A batched call captured into a CUDA graph on the first gridder's
    stream and replayed twice does what two batched calls do."""
    import torch
    jobs = make_jobs(seed=3, njobs=5)
    dv = [torch.from_numpy(np.frombuffer(j["vis"].tobytes(), np.uint8).copy()
                           ).cuda() for j in jobs]
    ref = gridders_for(jobs, precision, 0, False)
    for _ in range(2):
        hpg_b200.grid_visibilities_batch(ref, dv, on_device=True)
    ref[0].fence()
    gs = gridders_for(jobs, precision, 0, False)
    hpg_b200.grid_visibilities_batch(gs, dv, on_device=True)  # buffers
    gs[0].fence()
    for g in gs:
        g.reset_grid()
    with gs[0].capture() as graph:
        hpg_b200.grid_visibilities_batch(gs, dv, on_device=True)
    for _ in range(2):
        graph.launch()
    gs[0].fence()
    tol = 1e-12 if precision == abi.PRECISION_FP64 else 1e-6
    for a, b, job in zip(ref, gs, jobs):
        if len(job["vis"]):
            assert rel_norm(b.grid_values(), a.grid_values()) <= tol
        np.testing.assert_allclose(b.grid_weights(), a.grid_weights(),
                                   rtol=1e-12)
    graph.close()
    for g in ref + gs:
        g.close()


def test_batch_errors(gpu):
    jobs = make_jobs(seed=4, njobs=3)
    gs = gridders_for(jobs, abi.PRECISION_MIXED, 0, False)
    vis = [j["vis"] for j in jobs]
    with pytest.raises(HpgError):  # a gridder twice
        hpg_b200.grid_visibilities_batch([gs[0], gs[1], gs[0]], vis)
    gs[1].set_precision(abi.PRECISION_FP64)
    with pytest.raises(HpgError):  # forms differ
        hpg_b200.grid_visibilities_batch(gs, vis)
    gs[1].set_precision(abi.PRECISION_MIXED)
    other = Gridder.create(0, 0, 10, None, (64, 64, 2, 1), (0.05, 0.05),
                           [[0, 1], [2, 3]], [[0, 1], [2, 3]])
    with pytest.raises(HpgError):  # Mueller tables differ (and no CF)
        hpg_b200.grid_visibilities_batch([gs[0], other], vis[:2])
    odd = Gridder.create(0, 0, 10, None, (65, 64, 2, 1), (0.05, 0.05), MI,
                         MI)
    odd.set_precision(abi.PRECISION_MIXED)
    odd.set_convolution_function(CFArray(8, jobs[0]["cf_extents"],
                                         jobs[0]["cf_values"]))
    odd.set_model(np.zeros((1, 2, 64, 65), np.complex128))
    for g, job in zip(gs, jobs):
        g.set_model(job["model"])
    with pytest.raises(HpgError) as e:  # odd width: no FP32 model tensor map
        hpg_b200.grid_visibilities_batch([gs[0], odd], [vis[0], vis[0][:0]],
                                         do_degrid=True)
    assert "16-byte" in str(e.value)
    odd.close()
    with pytest.raises(HpgError) as e:  # a batch beyond its gridder's size
        hpg_b200.grid_visibilities_batch(
            gs, [vis[0], np.concatenate([vis[1]] * 3), vis[2]])
    assert e.value.type == "ExcessiveNumberVisibilities"
    hpg_b200.grid_visibilities_batch(gs, vis)  # still usable
    gs[0].fence()
    other.close()
    for g in gs:
        g.close()
