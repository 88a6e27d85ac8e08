"""Visibility sharding across ranks, on CPU: two gloo ranks each grid their
shard with the oracle and sum the grids; the result must equal one process
gridding the whole batch (to FP64 summation order, 1e-12)."""
import os
import socket

import numpy as np
import pytest

from hpg_b200 import distributed as D
from hpg_b200 import workloads


def test_shard_bounds_cover_exactly():
    for n in (0, 1, 5, 7, 1000):
        for world in (1, 2, 3, 8):
            bounds = [D.shard_bounds(n, world, r) for r in range(world)]
            assert bounds[0][0] == 0 and bounds[-1][1] == n
            for (a0, b0), (a1, b1) in zip(bounds, bounds[1:]):
                assert b0 == a1
            sizes = [b - a for a, b in bounds]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        D.shard_bounds(10, 2, 2)
    with pytest.raises(ValueError):
        D.shard_bounds(-1, 2, 0)


def _config():
    return workloads.full_pol_config(900, grid=64, oversampling=8,
                                     supports=(2, 4), seed=31)


def _oracle(cfg):
    from oracle import oracle as O
    return O.Oracle(cfg["grid_size"], cfg["grid_scale"], cfg["mueller"],
                    cfg["conj_mueller"], cfg["oversampling"],
                    cfg["cf_extents"], cfg["cf_values"])


def _worker(rank, world, port, queue):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    try:
        from datetime import timedelta
        dist.init_process_group("gloo", rank=rank, world_size=world,
                                timeout=timedelta(seconds=60))
        cfg = _config()

        def grid_shard(vis_shard):
            o = _oracle(cfg)
            o.grid_visibilities(vis_shard)
            return o.grid, o.weights

        grid, weights = D.grid_sharded(grid_shard, cfg["vis"])
        queue.put((rank, grid, weights))
        dist.destroy_process_group()
    except Exception as e:  # reported to the parent, which fails the test
        queue.put((rank, repr(e), None))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_two_rank_sharded_gridding_matches_one_process(oracle_lib):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, queue))
             for r in range(2)]
    for p in procs:
        p.start()
    results = {}
    for _ in range(2):
        rank, grid, weights = queue.get(timeout=180)
        assert not isinstance(grid, str), grid
        results[rank] = (grid, weights)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    cfg = _config()
    o = _oracle(cfg)
    o.grid_visibilities(cfg["vis"])
    for rank in (0, 1):
        grid, weights = results[rank]
        assert np.abs(o.grid).max() > 0
        assert np.linalg.norm(grid - o.grid) <= 1e-12 * np.linalg.norm(o.grid)
        np.testing.assert_allclose(weights, o.weights, rtol=1e-12)


def _device_worker(rank, world, port, queue, precision):
    """One rank: its own device gridder on cuda:0, its shard, the grids and
    weights summed over gloo."""
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    try:
        from datetime import timedelta
        from hpg_b200 import CFArray, Gridder
        dist.init_process_group("gloo", rank=rank, world_size=world,
                                timeout=timedelta(seconds=120))
        cfg = _config()

        def grid_shard(vis_shard):
            g = Gridder.create(0, 0, max(len(vis_shard), 1), None,
                               cfg["grid_size"], cfg["grid_scale"],
                               cfg["mueller"], cfg["conj_mueller"])
            g.set_precision(precision)
            g.set_convolution_function(CFArray(cfg["oversampling"],
                                               cfg["cf_extents"],
                                               cfg["cf_values"]))
            g.grid_visibilities(vis_shard)
            out = g.grid_values(), g.grid_weights()
            g.close()
            return out

        grid, weights = D.grid_sharded(grid_shard, cfg["vis"])
        queue.put((rank, grid, weights))
        dist.destroy_process_group()
    except Exception as e:  # reported to the parent, which fails the test
        queue.put((rank, repr(e), None))


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "mixed"])
def test_two_rank_sharded_device_gridding(gpu, oracle_lib, precision):
    """The same sharding with the device gridder on every rank (two
    processes on one GPU, no kernel waits on another rank; the grids meet
    in a gloo all-reduce of their complex128 arrays): equal to the oracle's
    gridding of the whole batch (1e-12 FP64, 1e-6 mixed)."""
    import multiprocessing as mp
    from hpg_b200 import abi
    prec = abi.PRECISION_FP64 if precision == 0 else abi.PRECISION_MIXED
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_device_worker, args=(r, 2, port, queue, prec))
             for r in range(2)]
    for p in procs:
        p.start()
    results = {}
    for _ in range(2):
        rank, grid, weights = queue.get(timeout=300)
        assert not isinstance(grid, str), grid
        results[rank] = (grid, weights)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    cfg = _config()
    o = _oracle(cfg)
    o.grid_visibilities(cfg["vis"])
    tol = 1e-12 if precision == 0 else 1e-6
    for rank in (0, 1):
        grid, weights = results[rank]
        assert np.linalg.norm(grid - o.grid) <= tol * np.linalg.norm(o.grid)
        np.testing.assert_allclose(weights, o.weights, rtol=1e-12)
