"""The tiled kernel's bounded waits: a wait that runs out ends the launch
with an error status that the next fence reports, and the gridder stays
usable.

The failure is made on the host side of the kernel's contract, never by a
fault: a test hook tells the grid-row-0 CTA that takes one visibility (a
position in the tile-sorted batch) not to issue its bulk copies, so the mbarrier phase that announces them never completes (a
flag that nothing sets).  With a 20 ms wait limit the waiting warps give up,
set the CTA's abort flag, and every role winds down through its barriers;
the peers of the cluster give up on that CTA's partial sums the same way.
Then the hook is cleared and the same batch grids as the oracle's.
"""
import time

import numpy as np
import pytest

from hpg_b200 import CFArray, Gridder, HpgError, abi, workloads

pytestmark = pytest.mark.gpu


def rel_norm(a, b):
    return np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel())


@pytest.mark.parametrize("degrid", [True, False], ids=["degrid+grid", "grid"])
@pytest.mark.parametrize("precision", [abi.PRECISION_FP64, abi.PRECISION_MIXED],
                         ids=["fp64", "mixed"])
def test_wait_timeout_reported_and_recovered(gpu, oracle_lib, precision,
                                             degrid):
    O = oracle_lib
    cfg = workloads.full_pol_config(3000, grid=256, oversampling=16,
                                    supports=(4, 6, 8, 10), seed=7, grad=0.3)
    vis = cfg["vis"]
    g = Gridder.create(0, 0, len(vis), None, cfg["grid_size"],
                       cfg["grid_scale"], cfg["mueller"], cfg["conj_mueller"])
    g.set_precision(precision)
    g.set_gridding_kernel(abi.KERNEL_TILED)
    g.set_convolution_function(CFArray(cfg["oversampling"], cfg["cf_extents"],
                                       cfg["cf_values"]))
    g.set_model(cfg["model"])
    run = g.degrid_grid_visibilities if degrid else g.grid_visibilities

    g.set_wait_limit(0.02)
    g.debug_withhold_copy(5)
    t0 = time.perf_counter()
    run(vis)
    with pytest.raises(HpgError) as e:
        g.fence()
    assert e.value.type == "Other"
    assert "wait" in str(e.value)
    assert time.perf_counter() - t0 < 10.0
    g.fence()  # the status was reported once and cleared

    g.debug_withhold_copy(-1)
    g.set_wait_limit(0.5)
    g.reset_grid()
    run(vis)
    g.fence()
    o = O.Oracle(cfg["grid_size"], cfg["grid_scale"], cfg["mueller"],
                 cfg["conj_mueller"], cfg["oversampling"], cfg["cf_extents"],
                 cfg["cf_values"])
    o.set_model(cfg["model"])
    o.grid_visibilities(vis, do_degrid=degrid)
    assert rel_norm(g.grid_values(), o.grid) <= 1e-6
    np.testing.assert_allclose(g.grid_weights(), o.weights, rtol=1e-12)
    g.close()


def test_wait_limit_arguments(gpu):
    g = Gridder.create(0, 0, 1, None, (16, 16, 1, 1), (0.1, 0.1), [[0]],
                       [[0]])
    for bad in (0.0, -1.0, 61.0, float("nan")):
        with pytest.raises(HpgError):
            g.set_wait_limit(bad)
    with pytest.raises(HpgError):
        g.debug_withhold_copy(-2)
    g.set_wait_limit(1.0)
    g.debug_withhold_copy(-1)
    g.close()
