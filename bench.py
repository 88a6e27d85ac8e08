"""Benchmark of the gridding / degridding hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--precision both|mixed|fp64] [--nvis 10000000]

Workload (one "step"): degrid_grid_visibilities of one batch of 10M
four-polarization visibilities onto a 2048x2048x4x1 complex128 grid with a
dense 4x4 Mueller matrix (16 CF planes), 8 w-plane CF groups with supports
8..32 (9..33 taps) at oversampling 128, starting from a complex128 N(0,1)
model.  All inputs are seeded synthetic data with those shapes.

Printed (rank 0, one JSON line): Mvis/s of the mixed form with inputs
resident in HBM ("value"; the FP64 form is timed beside it under "forms"),
the same through the public API with pinned host input and a device->host
read of the weights after every step, pipelined as a caller streaming
batches would ("e2e"), the HBM roofline of the tiled kernel (its
algorithmic bytes over its CUDA-event time) and of the whole step, the error
of the mixed grid against the FP64 grid at full size, the CPU baseline
(threaded CPU restatement on a bounded sample) and the SM clocks sampled
during the timed region.

Under torchrun (N > 1) every rank runs its own replica of the workload on its
GPU (weak scaling); the step time is the maximum over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mvis/s grid+degrid (degrid_grid_visibilities), 2048^2x4 pol, 10M vis"
UNIT = "Mvis/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--precision", default="both",
                   choices=["both", "mixed", "mixed-comp", "fp64"],
                   help="both: the mixed form is the headline, the "
                        "compensated mixed form and the FP64 form are timed "
                        "beside it")
    p.add_argument("--nvis", type=int, default=10_000_000)
    p.add_argument("--grid", type=int, default=2048)
    p.add_argument("--oversampling", type=int, default=128,
                   help="CF oversampling (smaller values shrink the CF table "
                        "for profiling captures; per-visibility work is "
                        "unchanged)")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-autotune", dest="autotune", action="store_false",
                   help="skip the (untimed) autotuning of the tiled plan")
    p.add_argument("--cpu-seconds", type=float, default=12.0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--workload", default="full-pol",
                   choices=["full-pol", "adjoint", "batch"],
                   help="full-pol: the headline degrid+grid step; adjoint: "
                        "one gradient step of the differentiable-imaging "
                        "workload (D then D^H on a 4096^2 x 2 grid, 32 CF "
                        "groups of supports 8..64, FP64 operators); batch: "
                        "64 uneven gridding jobs, one launch per "
                        "polarization class, against one launch per job")
    p.add_argument("--jobs", type=int, default=64)
    return p.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,"
              "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"),
                stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax),
                "samples": len(sm), "reasons": sorted(reasons)}


def make_workload(args, seed_offset, device):
    import torch
    from hpg_b200 import workloads
    p = workloads.full_pol_params(supports=workloads.FULL_POL_SUPPORTS,
                                  oversampling=args.oversampling,
                                  seed=20261204 + seed_offset)
    rng = p["rng"]
    grid_size = (args.grid, args.grid, 4, 1)
    vis = workloads.visibilities(args.nvis, 4, grid_size, p["grid_scale"],
                                 p["freq"], rng, w_frac=0.3,
                                 ngroups=len(p["supports"]))
    ext, vals = workloads.separable_cf_torch(p["supports"], p["oversampling"],
                                             p["mueller_factors"], device,
                                             w_phases=p["w_phases"])
    g = torch.Generator(device=device).manual_seed(7 + seed_offset)
    model = torch.complex(
        torch.randn((1, 4, args.grid, args.grid), generator=g, device=device,
                    dtype=torch.float64),
        torch.randn((1, 4, args.grid, args.grid), generator=g, device=device,
                    dtype=torch.float64))
    return dict(p=p, grid_size=grid_size, vis=vis, cf_extents=ext,
                cf_values=vals, model=model)


# DRAM bytes (read + write) of one tiled-kernel launch, from an ncu capture
# of 200k visibilities of this workload at CF oversampling 64 (mixed form:
# 15.75 GB, of which 0.67 GB are the model and grid passes; FP64 form:
# 16.04 GB, 0.81 GB), scaled to a launch by the visibility count.
TRAFFIC_PER_VIS_MIXED = (15.754e9 - 0.671e9) / 200_000
TRAFFIC_PER_VIS_FP64 = (16.036e9 - 0.805e9) / 200_000


def kernel_traffic(form, nvis, grid_elems):
    if form.startswith("mixed"):
        return TRAFFIC_PER_VIS_MIXED * nvis + grid_elems * (8 + 32)
    return TRAFFIC_PER_VIS_FP64 * nvis + grid_elems * (16 + 32)


def workload_name(args):
    return (f"full-pol degrid+grid {args.grid}x{args.grid}x4, 8 CF groups "
            f"(supports 8-32, os {args.oversampling}), dense 4x4 Mueller")


def config_of(args, world, precision):
    """The workload's config object, the same in both arms."""
    return {"workload": workload_name(args), "nvis": args.nvis,
            "grid": [args.grid, args.grid, 4, 1], "precision": precision,
            "l2": "inputs larger than L2 (CF 10 GB, visibilities 1.2 GB)",
            "parallelism": f"replicas x{world}"}


def taps_of(supports):
    return [s + 1 if s % 2 == 0 else s for s in supports]


def cpu_baseline(wl, target_s, nthreads=None):
    """Threaded CPU restatement (oracle) of the same step on a bounded
    sample of the same visibilities; returns (Mvis/s, sample, threads)."""
    from oracle import oracle as O
    p = wl["p"]
    nthreads = nthreads or O.num_threads()
    cf_host = [v.cpu().numpy() for v in wl["cf_values"]]
    model = wl["model"].cpu().numpy()
    o = O.Oracle(wl["grid_size"], p["grid_scale"], p["mueller"],
                 p["conj_mueller"], p["oversampling"], wl["cf_extents"],
                 cf_host)
    o.set_model(model)
    vis = wl["vis"]
    n = 2000
    t0 = time.perf_counter()
    o.grid_visibilities(vis[:n], do_degrid=True, nthreads=nthreads)
    dt = time.perf_counter() - t0
    n2 = int(min(len(vis) - n, max(n, target_s / max(dt / n, 1e-9))))
    t0 = time.perf_counter()
    res = o.grid_visibilities(vis[n:n + n2], do_degrid=True, return_vis=True,
                              nthreads=nthreads)
    dt2 = time.perf_counter() - t0
    # what the oracle computed on the sample: the parity check of the
    # device against it grids the same n + n2 visibilities
    oracle_out = dict(n_warm=n, n_sample=n2, residuals=res["vis"],
                      grid=o.grid, weights=o.weights)
    return n2 / dt2 / 1e6, n2, dt2, nthreads, oracle_out


def device_parity(g, vis, ref, form):
    """The device's degrid+grid of the CPU-baseline sample (a fresh grid,
    the same n_warm + n_sample visibilities) against the oracle's results:
    relative norm errors of the grid, the weights and the residual
    visibilities, and the fraction of bit-exact residuals."""
    from hpg_b200 import abi
    g.reset_grid()
    nw, ns = ref["n_warm"], ref["n_sample"]
    g.degrid_grid_visibilities(vis[:nw])
    fut = g.degrid_grid_get_residual_visibilities(vis[nw:nw + ns])
    g.fence()
    res = fut.get()["vis"]
    grid, wgt = g.grid_values(), g.grid_weights()

    def rel(a, b):
        return float(np.linalg.norm((a - b).ravel()) /
                     np.linalg.norm(b.ravel()))
    out = {"visibilities": nw + ns,
           "grid_rel": rel(grid, ref["grid"]),
           "weights_rel": rel(wgt, ref["weights"]),
           "residual_rel": rel(res.astype(np.complex128),
                               ref["residuals"].astype(np.complex128)),
           "residual_bit_exact": float(np.mean(np.all(
               res == ref["residuals"], axis=1)))}
    tol = 1e-6
    out["within_tolerance"] = bool(out["grid_rel"] <= tol and
                                   out["residual_rel"] <= tol and
                                   out["weights_rel"] <= 1e-12)
    del abi
    return out


def run_reference(args, rank):
    """The reference's CPU implementation of the path (its Kokkos
    Serial/OpenMP build is not buildable here: the CPU restatement stands in)
    on the host cores, on this arm's workload and metric."""
    if rank != 0:
        return
    import torch
    from oracle import oracle as O
    dev = torch.device("cuda", 0) if torch.cuda.is_available() else torch.device("cpu")
    wl = make_workload(args, 0, dev)
    nthreads = O.num_threads()
    p = wl["p"]
    cf_host = [v.cpu().numpy() for v in wl["cf_values"]]
    model = wl["model"].cpu().numpy()
    del wl["cf_values"]
    o = O.Oracle(wl["grid_size"], p["grid_scale"], p["mueller"],
                 p["conj_mueller"], p["oversampling"], wl["cf_extents"], cf_host)
    o.set_model(model)
    vis = wl["vis"]
    # bounded sample per step: ~args.cpu_seconds / (warmup + steps)
    n = 1000
    t0 = time.perf_counter()
    o.grid_visibilities(vis[:n], do_degrid=True, nthreads=nthreads)
    per_vis = (time.perf_counter() - t0) / n
    per_step = max(2.0, 60.0 / max(args.steps + args.warmup, 1))
    n_step = int(max(1000, min(len(vis), per_step / per_vis)))
    off = n
    for _ in range(args.warmup):
        o.grid_visibilities(vis[off:off + n_step], do_degrid=True, nthreads=nthreads)
        off = (off + n_step) % max(len(vis) - n_step, 1)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        o.grid_visibilities(vis[off:off + n_step], do_degrid=True, nthreads=nthreads)
        times.append(time.perf_counter() - t0)
        off = (off + n_step) % max(len(vis) - n_step, 1)
    value = n_step * len(times) / sum(times) / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": config_of(args, args.gpus, "mixed"
                            if args.precision == "both" else args.precision),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthreads,
                         "kind": "port",
                         "sample": f"{n_step} visibilities per step of the "
                                   f"{args.nvis}-visibility batch"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


ADJ_SUPPORTS = tuple(8 + (56 * k) // 31 for k in range(32))  # 8 .. 64


def run_adjoint(args):
    """Gradient step of L = sum w |D(G) - V|^2 on one GPU: y = D(G) (FP64
    degridding), r = w (y - V), dL/dG = 2 D^H(r), through the tiled
    operators (hpgb_degrid_linear / hpgb_degrid_adjoint).  Workload: a
    4096 x 4096 x 2 grid (diagonal Mueller), 32 w-plane CF groups of
    supports 8..64 at oversampling 128, args.nvis visibilities (seeded
    synthetic data of those shapes; G = point sources plus N(0, 0.01)
    noise).  Prints one JSON line: Mvis/s of the step, each operator's
    time and its HBM roofline (CF slice bytes per visibility, grid bytes per
    pass)."""
    import ctypes
    import torch
    import hpg_b200
    from hpg_b200 import CFArray, Gridder, abi, workloads
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    hpg_b200.load()
    side = 4096
    npol = 2
    rng = np.random.default_rng(20261207)
    supports = ADJ_SUPPORTS
    os_ = args.oversampling
    mf = np.ones(npol, np.complex128)
    w_phases = [0.01 * k for k in range(len(supports))]
    ext, vals = workloads.separable_cf_torch(supports, os_, mf, dev,
                                             w_phases=w_phases)
    gs = (side, side, npol, 1)
    scale = (0.0476591, 0.0476591)
    vis = workloads.visibilities(args.nvis, npol, gs, scale, 1.4e9, rng,
                                 w_frac=0.3, ngroups=len(supports))
    mi = [[0, -1], [-1, 1]]
    g = Gridder.create(0, 0, args.nvis, None, gs, scale, mi, mi)
    g.set_convolution_function(CFArray(os_, ext, vals), on_device=True)
    del vals
    torch.cuda.empty_cache()
    dvis = torch.from_numpy(vis.view(np.uint8)).to(dev)
    gen = torch.Generator(device=dev).manual_seed(11)
    G = (torch.randn((1, npol, side, side), generator=gen, device=dev,
                     dtype=torch.float64) * 0.01 + 0j)
    pts = torch.randint(0, side, (1000, 2), generator=gen, device=dev)
    G[0, :, pts[:, 1], pts[:, 0]] += 1.0
    V = torch.from_numpy(vis["vis"].astype(np.complex128)).to(dev)
    W = torch.from_numpy(vis["weights"].astype(np.float64)).to(dev)
    y = torch.empty((args.nvis, npol), dtype=torch.complex128, device=dev)
    grad = torch.zeros_like(G)
    lib = abi.load()
    stream = torch.cuda.ExternalStream(g.stream, device=dev)
    P = ctypes.c_void_p

    def step(ev=None):
        abi.check(lib.hpgb_degrid_linear(g._h, P(dvis.data_ptr()), args.nvis,
                                         npol, P(G.data_ptr()),
                                         P(y.data_ptr())))
        if ev:
            ev[1].record(stream)
        with torch.cuda.stream(stream):
            r = (y - V) * (2.0 * W)
            grad.zero_()
            if ev:
                ev[2].record(stream)
            abi.check(lib.hpgb_degrid_adjoint(g._h, P(dvis.data_ptr()),
                                              args.nvis, npol,
                                              P(r.data_ptr()),
                                              P(grad.data_ptr())))
        return r

    for _ in range(args.warmup):
        step()
    g.fence()
    torch.cuda.synchronize()
    t_d, t_dh, t_step = [], [], []
    for _ in range(args.steps):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        ev[0].record(stream)
        r = step(ev)
        ev[3].record(stream)
        ev[3].synchronize()
        t_d.append(ev[0].elapsed_time(ev[1]))
        t_dh.append(ev[2].elapsed_time(ev[3]))
        t_step.append(ev[0].elapsed_time(ev[3]))
        del r
    assert g.last_gridding_kernel() == abi.KERNEL_TILED
    peak, peak_kind = peaks()
    taps = np.asarray(taps_of(supports), np.int64)[
        vis["cf_index"][:, 1].astype(np.int64)]
    cf_bytes = int((taps * taps).sum()) * 1 * 8 * npol  # one plane per row
    grid_bytes = side * side * npol * 16
    vals_bytes = args.nvis * npol * 16
    # algorithmic bytes per operator launch: the CF slices once, the grid
    # once (D reads the model; D^H reads and writes the gradient), the
    # visibility values once
    b_d = cf_bytes + grid_bytes + vals_bytes
    b_dh = cf_bytes + 2 * grid_bytes + vals_bytes
    ms_d, ms_dh = statistics.median(t_d), statistics.median(t_dh)
    ms_step = statistics.median(t_step)
    line = {
        "metric": "Mvis/s loss-gradient step (D then D^H), 4096^2x2, "
                  "supports 8-64",
        "value": args.nvis / (ms_step * 1e-3) / 1e6, "unit": "Mvis/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_step, "higher_is_better": True, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"differentiable degridding 4096x4096x2, 32 "
                               f"CF groups (supports 8-64, os {os_}), "
                               f"diagonal Mueller",
                   "nvis": args.nvis},
        "operators": {
            "D": {"ms": ms_d, "gbs": b_d / (ms_d * 1e-3) / 1e9,
                  "frac": b_d / (ms_d * 1e-3) / 1e9 / peak,
                  "algorithmic_bytes": b_d},
            "D^H": {"ms": ms_dh, "gbs": b_dh / (ms_dh * 1e-3) / 1e9,
                    "frac": b_dh / (ms_dh * 1e-3) / 1e9 / peak,
                    "algorithmic_bytes": b_dh},
        },
        "cf_bytes_per_vis": cf_bytes / args.nvis,
        "peak": peak, "peak_kind": peak_kind,
    }
    print(json.dumps(line), flush=True)
    g.close()


def run_batch(args):
    """The batched, uneven workload: args.jobs independent gridding jobs,
    each with a grid side log-uniform in [256, 2048], 1, 2 or 4
    polarizations (diagonal Mueller), a batch log-uniform in [10k, 2M]
    visibilities (uv uniform in the disk), 1..16 CF groups with supports
    drawn from {8, 16, 32, 64} at oversampling 64; mixed form.  One step
    grids every job's batch: the jobs of each polarization count go to one
    hpgb_grid_visibilities_batch call, which takes one persistent tiled
    launch per group of its gridders with the same CF support class and
    tile side, device-resident inputs.  The same step is timed with one call per job
    (one tiled launch each) beside it.  Prints one JSON line: Mvis/s of both, and the
    batched launches' HBM roofline (records + CF slices once per visibility
    + grid read/write per job)."""
    import torch
    import hpg_b200
    from hpg_b200 import CFArray, Gridder, abi, workloads
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    hpg_b200.load()
    rng = np.random.default_rng(20261206)
    os_ = 64
    scale = (0.0476591, 0.0476591)
    jobs = []
    for j in range(args.jobs):
        side = int(np.exp(rng.uniform(np.log(256), np.log(2048)))) & ~1
        npol = int(rng.choice([1, 2, 4]))
        nvis = int(np.exp(rng.uniform(np.log(1e4), np.log(2e6))))
        ngroups = int(rng.integers(1, 17))
        supports = [int(x) for x in rng.choice([8, 16, 32, 64], ngroups)]
        mi = [[r if c == r else -1 for c in range(npol)] for r in range(npol)]
        gs = (side, side, npol, 1)
        ext, vals = workloads.separable_cf_torch(
            supports, os_, np.ones(npol) + 0.1j * rng.standard_normal(npol),
            dev)
        g = Gridder.create(0, 0, nvis, None, gs, scale, mi, mi)
        g.set_precision(abi.PRECISION_MIXED)
        g.set_convolution_function(CFArray(os_, ext, vals), on_device=True)
        del vals
        vis = workloads.visibilities(nvis, npol, gs, scale, 1.4e9, rng,
                                     ngroups=ngroups)
        dvis = torch.from_numpy(vis.view(np.uint8)).to(dev)
        taps = np.asarray(taps_of(supports), np.int64)[
            vis["cf_index"][:, 1].astype(np.int64)]
        jobs.append(dict(g=g, dvis=dvis, npol=npol, nvis=nvis, side=side,
                         max_support=max(supports),
                         bytes=int(len(vis) * vis.dtype.itemsize +
                                   (taps * taps).sum() * npol * 8 +
                                   2 * side * side * npol * 16)))
        del vis
    torch.cuda.empty_cache()
    # one batched call per polarization class (the library splits each by
    # the gridders' widest CF and own tile side into launches)
    classes = {}
    for job in jobs:
        classes.setdefault(job["npol"], []).append(job)
    total_vis = sum(j["nvis"] for j in jobs)
    total_bytes = sum(j["bytes"] for j in jobs)
    def batched(groups):
        for cls in groups.values():
            hpg_b200.grid_visibilities_batch(
                [j["g"] for j in cls], [j["dvis"] for j in cls],
                on_device=True)

    def per_job():
        for job in jobs:
            job["g"].grid_visibilities(job["dvis"], on_device=True)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        for job in jobs:
            job["g"].fence()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record()
        for _ in range(args.steps):
            fn()
        for job in jobs:  # every gridder's work before the end event
            e = torch.cuda.Event()
            e.record(torch.cuda.ExternalStream(job["g"].stream, device=dev))
            torch.cuda.current_stream().wait_event(e)
        ev1.record()
        ev1.synchronize()
        return ev0.elapsed_time(ev1) / args.steps

    # each class's launch runs on the stream of its first gridder, so the
    # classes may overlap; the step ends when every gridder's work has
    ms_batched = timed(lambda: batched(classes))
    # each polarization class alone: its batched call against its jobs'
    # own calls
    per_class = {}

    def kernel_ms(cls):
        """Summed CUDA-event time of the tiled launches recorded since the
        last call, over the class's gridders (a batched call records its
        launches on the first gridders of its groups; they may overlap)."""
        tot, launches = 0.0, 0
        for j in cls:
            ms, n = j["g"].tiled_kernel_time()
            tot += ms
            launches += n
        return tot, launches

    for k, cls in classes.items():
        one = {k: cls}
        for j in cls:
            j["g"].profile_tiled_kernel(True)
        kernel_ms(cls)
        mb = timed(lambda: batched(one))
        kb, nl = kernel_ms(cls)
        kb /= args.steps + args.warmup
        nl //= args.steps + args.warmup
        for j in cls:
            j["g"].profile_tiled_kernel(False)
        # (the per-job launches' event times are not summed: a launch on
        # one gridder's stream waits inside its events for the SMs that
        # the other gridders' launches hold)
        ms = timed(lambda: [j["g"].grid_visibilities(j["dvis"], on_device=True)
                            for j in cls])
        per_class[f"{k}pol"] = {"jobs": len(cls),
                                "vis": sum(j["nvis"] for j in cls),
                                "batched_ms": mb, "per_job_ms": ms,
                                "batched_kernel_ms_sum": kb,
                                "batched_launches": nl}
    for job in jobs:
        job["g"].set_gridding_kernel(abi.KERNEL_TILED)
    ms_single = timed(per_job)
    peak, peak_kind = peaks()
    line = {
        "metric": "Mvis/s gridding of 64 uneven jobs (batched launches)",
        "value": total_vis / (ms_batched * 1e-3) / 1e6, "unit": "Mvis/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_batched, "higher_is_better": True,
        "dtype": "f32-mixed", "data": "synthetic",
        "config": {"workload": f"{args.jobs} gridding jobs: side 256-2048 "
                               f"log-uniform, 1/2/4 pol diagonal, 10k-2M "
                               f"vis, 1-16 CF groups of supports "
                               f"{{8,16,32,64}}, os {os_}",
                   "total_vis": total_vis,
                   "batch_calls": len(classes),
                   "jobs_per_call": {f"{k}pol": len(v)
                                     for k, v in classes.items()},
                   "launches": sum(c["batched_launches"]
                                   for c in per_class.values())},
        "per_class": per_class,
        "per_job_launches": {"value": total_vis / (ms_single * 1e-3) / 1e6,
                             "ms_per_step": ms_single},
        "roofline": {"bound": "hbm", "achieved": total_bytes /
                     (ms_batched * 1e-3) / 1e9, "peak": peak,
                     "unit": "GB/s",
                     "frac": total_bytes / (ms_batched * 1e-3) / 1e9 / peak,
                     "peak_kind": peak_kind,
                     "algorithmic_bytes_per_step": total_bytes,
                     "scope": "whole step (sort, descriptors, tiled launch)"},
    }
    print(json.dumps(line), flush=True)
    for job in jobs:
        job["g"].close()


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.workload == "adjoint":
        run_adjoint(args)
        return
    if args.workload == "batch":
        run_batch(args)
        return
    import torch
    import torch.distributed as dist
    import hpg_b200
    from hpg_b200 import CFArray, Gridder, abi, workloads

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=dev)
    hpg_b200.load()

    wl = make_workload(args, rank, dev)
    p = wl["p"]
    g = Gridder.create(local_rank, 0, args.nvis, None, wl["grid_size"],
                       p["grid_scale"], p["mueller"], p["conj_mueller"])
    g.set_convolution_function(CFArray(p["oversampling"], wl["cf_extents"],
                                       wl["cf_values"]), on_device=True)
    g.set_model(wl["model"], on_device=True)
    cpu_wl = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu_wl = wl
    else:
        del wl["cf_values"]
        torch.cuda.empty_cache()

    vis = wl["vis"]
    dvis = torch.from_numpy(vis.view(np.uint8)).to(dev)
    hvis = torch.from_numpy(vis.view(np.uint8)).pin_memory()
    hvis_np = hvis.numpy().view(vis.dtype)
    stream = torch.cuda.ExternalStream(g.stream, device=dev)

    def step_device():
        g.degrid_grid_visibilities(dvis, on_device=True)

    # the weights in device memory (the reference's grid_weights_ptr()),
    # read back after every end-to-end step without fencing the gridder
    class _DeviceArray:
        def __init__(self, ptr, n):
            self.__cuda_array_interface__ = {
                "shape": (n,), "typestr": "<f8", "data": (ptr, False),
                "version": 3}
    wdev = torch.as_tensor(_DeviceArray(*g.grid_weights_ptr()), device=dev)
    wpin = [torch.empty(wdev.numel(), dtype=torch.float64).pin_memory()
            for _ in range(2)]
    wev = [torch.cuda.Event() for _ in range(2)]

    def run_e2e(k):
        """k steps through the public API, pipelined as a caller streaming
        batches would: each step queues its batch (pinned host memory; the
        host->device copy is part of the call and overlaps the previous
        step's work) and a device->host copy of the weights behind it on the
        gridder's stream; the host reads step j's weights once step j + 1 is
        queued.  Returns the weight sums read."""
        sums = []
        for j in range(k):
            g.degrid_grid_visibilities(hvis_np)
            with torch.cuda.stream(stream):
                wpin[j % 2].copy_(wdev, non_blocking=True)
                wev[j % 2].record(stream)
            if j > 0:
                wev[(j - 1) % 2].synchronize()
                sums.append(float(wpin[(j - 1) % 2].sum()))
        wev[(k - 1) % 2].synchronize()
        sums.append(float(wpin[(k - 1) % 2].sum()))
        return sums

    def timed(fn, k):
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        g.fence()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(k):
            fn()
        ev1.record(stream)
        ev1.synchronize()
        g.fence()
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1)
        if world > 1:
            t = torch.tensor([ms], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
            dist.barrier()
        return ms

    taps = taps_of(p["supports"])
    grid_elems = int(np.prod(wl["grid_size"]))
    b_alg = workloads.algorithmic_bytes(vis, 4, taps, 16, grid_elems, 3)
    # the tiled kernel's share: CF slices + model read + grid read/write (the
    # visibility records are read by the sort and descriptor kernels)
    b_kernel = b_alg - len(vis) * vis.dtype.itemsize
    peak, peak_kind = peaks()
    total_vis = args.nvis * world

    forms = (["mixed", "mixed-comp", "fp64"] if args.precision == "both"
             else [args.precision])
    results = {}
    plans = {}
    clock_summary = None

    def use_form(form, plan=None):
        """Arithmetic form: "mixed" (FP32 products and tiles), "mixed-comp"
        (the same with compensated two-sum tile pairs) or "fp64"."""
        g.set_precision(hpg_b200.PRECISION_FP64 if form == "fp64"
                        else hpg_b200.PRECISION_MIXED)
        comp = abi.COMPENSATED_ON if form == "mixed-comp" else 0
        plan = plan or {}
        g.set_tiled_plan(plan.get("ring_parts", 0), plan.get("chunk_vis", 0),
                         plan.get("tile_side", 0), comp)

    for form in forms:
        use_form(form)
        # untimed set-up: the autotuner picks the tiled plan on this batch
        plan = None
        if args.autotune:
            g.autotune_tiled(dvis, on_device=True)
            plan = g.tiled_plan()
        plans[form] = plan
        for _ in range(args.warmup):
            step_device()
        g.fence()
        g.tiled_kernel_time()
        g.profile_tiled_kernel(True)
        clocks = ClockSampler(local_rank)
        clocks.start()
        launches0 = g.kernel_launches()
        ms = timed(step_device, args.steps)
        launches = g.kernel_launches() - launches0
        csum = clocks.stop()
        g.profile_tiled_kernel(False)
        kms, kcount = g.tiled_kernel_time()
        ms_step = ms / args.steps
        k_avg = kms / kcount if kcount else None
        results[form] = {
            "value": total_vis / (ms_step * 1e-3) / 1e6,
            "ms_per_step": ms_step,
            "kernel_ms": k_avg, "kernel_launches": kcount,
            "gpu_launches": launches,
            "step_gbs": b_alg / (ms_step * 1e-3) / 1e9,
            "kernel_gbs": (b_kernel / (k_avg * 1e-3) / 1e9) if k_avg else None,
            "clocks": csum,
            "tiled_plan": plan if plan else "automatic",
        }
        if form == forms[0]:
            clock_summary = csum

    head = results[forms[0]]

    # end to end, every form: at least 10 pipelined steps, so that the first
    # step's unoverlapped copy and the last step's drain weigh little
    e2e_value = None
    e2e_steps = max(10, args.steps)
    if not args.no_e2e:
        for form in forms:
            use_form(form, plans.get(form))
            run_e2e(2)
            ms_e2e = timed(lambda: run_e2e(e2e_steps), 1)
            results[form]["e2e"] = total_vis / (ms_e2e / e2e_steps * 1e-3) / 1e6
            results[form]["e2e_steps"] = e2e_steps
        e2e_value = results[forms[0]]["e2e"]

    # full-size error of the mixed forms against the FP64 form (one step each
    # from a zero grid; the FP64 form is checked against the CPU oracle by
    # the parity tests and the parity field)
    mixed_err = None
    if "mixed" in results and "fp64" in results:
        grids = {}
        for form in [f for f in ("fp64", "mixed", "mixed-comp") if f in results]:
            use_form(form, plans.get(form))
            g.reset_grid()
            # the same step, returning the residual visibilities into a copy
            # of the batch
            dres = dvis.clone()
            g.degrid_grid_get_residual_visibilities(dres, on_device=True)
            g.fence()
            res = np.frombuffer(dres.cpu().numpy().tobytes(),
                                abi.visdata_dtype(4))["vis"]
            grids[form] = (g.grid_values(), g.grid_weights(), res)
            del dres
        gf, wf, rf = grids.pop("fp64")
        mixed_err = {}
        for form, (gm, wm, rm) in grids.items():
            mixed_err[form] = {
                "grid_rel": float(np.linalg.norm((gm - gf).ravel()) /
                                  np.linalg.norm(gf.ravel())),
                "weights_rel": float(np.linalg.norm(wm - wf) /
                                     np.linalg.norm(wf)),
                "residual_vis_rel": float(
                    np.linalg.norm((rm.astype(np.complex128) - rf).ravel()) /
                    np.linalg.norm(rf.astype(np.complex128).ravel())),
            }
        del grids, gf, rf

    cpu = None
    parity = None
    if cpu_wl is not None:
        try:
            v, n, dt, nt, oracle_out = cpu_baseline(cpu_wl, args.cpu_seconds)
            cpu = {"value": v, "unit": UNIT, "cores": nt, "kind": "port",
                   "sample": f"{n} visibilities of the same batch "
                             f"({dt:.1f} s, threaded CPU restatement)"}
        except Exception as e:  # reported, not hidden
            oracle_out = None
            cpu = {"value": None, "unit": UNIT, "cores": None, "kind": "port",
                   "sample": f"failed: {e}"}
        # the device on the same sample, from a fresh grid, every form
        if oracle_out is not None:
            parity = {}
            for form in forms:
                use_form(form, plans.get(form))
                parity[form] = device_parity(g, vis, oracle_out, form)

    if rank == 0:
        kernel_gbs = head["kernel_gbs"]
        line = {
            "metric": METRIC, "value": head["value"], "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": head["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if forms[0] == "fp64" else "f32-mixed",
            "data": "synthetic",
            "config": config_of(args, world, forms[0]),
            "forms": results,
            "mixed_over_fp64": ({f: results[f]["value"] /
                                 results["fp64"]["value"]
                                 for f in results if f != "fp64"}
                                if "fp64" in results else None),
            "mixed_vs_fp64_error": mixed_err,
            "e2e": {"value": e2e_value, "unit": UNIT,
                    "h2d_bytes_per_step": int(vis.nbytes),
                    "d2h_bytes_per_step": int(np.prod(wl["grid_size"][2:]) * 8)},
            "roofline": {"bound": "hbm", "kernel": "tiled_kernel",
                         "achieved": kernel_gbs, "peak": peak,
                         "unit": "GB/s",
                         "frac": kernel_gbs / peak if kernel_gbs else None,
                         "peak_kind": peak_kind,
                         "traffic": kernel_traffic(forms[0], args.nvis,
                                                   grid_elems),
                         "traffic_source": "ncu capture, 200k visibilities "
                                           "at CF oversampling 64, scaled by "
                                           "visibility count",
                         "algorithmic_bytes_per_launch": b_kernel,
                         "step_achieved": head["step_gbs"],
                         "step_frac": head["step_gbs"] / peak,
                         "algorithmic_bytes_per_step": b_alg},
            "cpu_baseline": cpu,
            "parity": parity,
            "clocks": clock_summary,
            "gpu_launches": head["gpu_launches"],
        }
        print(json.dumps(line), flush=True)
    # the pinned weight buffers were copied into on the gridder's stream;
    # torch's pinned-memory allocator records its release events on that
    # stream when they are freed, so they go before the stream does
    wpin.clear()
    wev.clear()
    wdev = None
    torch.cuda.synchronize()
    g.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
