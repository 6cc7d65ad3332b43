"""Benchmark of the sparse-grid interpolation hot path on B200.

Workload (one GPU): one adaptive d=59 grid of 1,000,000 nodes grown by seeded
random refinement (levels <= 7), TotalDof = 256, and 1,000,000 query points
(first half uniform in [0,1]^59, second half N(0.5, 0.05^2) clipped to [0,1]).
A step is one forward pass over all points.  The headline form is the batched
FP32 + compensated kernel (SGI_FP32C); the plain FP64 kernel (bit-identical to
the reference's gold path) is timed beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

With N > 1 (one process per GPU under torchrun) every rank replicates the grid
and evaluates its own 1M points (weak scaling, no collective on the data path).
`--impl reference` times the reference's own CPU code (oracle/_ref, compiled
from the reference sources) on the host cores over a bounded sample of points.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "hddm-solver-postprocessors_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

DIM, NNO, TD, NPTS = 59, 1_000_000, 256, 1_000_000
GRID_SEED, POINT_SEED = 4, 40
METRIC = "d=59 points/s: batched FP32+comp vs plain FP64 GPU @<=1e-7 rel err; %HBM peak"
WORKLOAD = "C4: d=59 adaptive grid, 1M nodes (levels<=7), TotalDof=256, 1M points (half U[0,1], half N(0.5,0.05^2))"


def env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def make_workload(npts=NPTS, seed_offset=0):
    import hddm_b200 as H
    t = time.time()
    hg = H.HostGrid.adaptive(DIM, NNO, TD, seed=GRID_SEED)
    X = H.gen_points(DIM, npts, kind=2, seed=POINT_SEED + seed_offset)
    return hg, X, time.time() - t


def alg_bytes(hg, info, npts, s_b):
    """SURVEY 8(d) algorithmic bytes of one launch (each grid counted once)."""
    idx, _ = hg.arrays()
    i = idx[:, :DIM]
    j = idx[:, DIM:]
    nz = (i != 0) | (j != 0)
    dims = np.broadcast_to(np.arange(DIM), i.shape)[nz].astype(np.int64)
    keys = (dims << 32) | (i[nz].astype(np.int64) << 16) | j[nz].astype(np.int64)
    szxps = int(np.unique(keys).size) + 1
    return (npts * DIM * 8 + npts * TD * 8 + info.nno * TD * s_b + info.ncoarse * TD * 4
            + 2 * info.nno * info.max_comps + 4 * szxps), szxps


# Random 1 KB row gathers from an L2-resident region measured 18.2G rows/s
# (18.7 TB/s) on this pool's B200s with 16-byte loads at 32 warps per SM
# (profiles/gather_roof_probe.md): the roof of a kernel whose work is one row
# gather per (point, active node) pair.
GATHER_PEAK_TBS = 18.7

# DRAM bytes (read + write) of one FP32C step of the default workload: the sum
# over the 16 fwd_f32d_kernel launches (node chunks of 64,768) of one forward
# call in an ncu capture (profiles/fwd_f32d_c4_traffic.md).
FP32C_STEP_DRAM_BYTES = 48.9e9


def gather_roof(mean_active, ms, grid, hg):
    """Row bytes the FP32C step gathers (one FP32 row per active pair, a lower
    bound) over the step time, against the measured gather peak."""
    info = grid.info
    row32 = info.ld * 4
    bytes_per_pair = row32  # lower bound: every pair reads at least its FP32 row
    b = mean_active * NPTS * bytes_per_pair
    ach = b / (ms * 1e-3) / 1e12
    return {"bound": "l2_gather", "achieved": ach, "peak": GATHER_PEAK_TBS, "unit": "TB/s",
            "frac": ach / GATHER_PEAK_TBS, "bytes_per_pair": bytes_per_pair,
            "note": "one FP32 row (TotalDof x 4 B) per active (point, node) pair over the step time; big "
                    "terms read their FP64 row (2x) and dropped terms read none"}


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        self.file.flush()
        rows = []
        for line in open(self.file.name):
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                try:
                    rows.append((float(f[1]), float(f[2]), f[5:9]))
                except ValueError:
                    pass
        os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = sorted(r[0] for r in rows)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[2][k].lower().startswith("active")})
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": max(r[1] for r in rows), "reasons": reasons,
                "samples": len(rows)}


def run_gpu(args):
    import torch
    import torch.distributed as dist

    import hddm_b200 as H

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    npts = args.points
    hg, X, t_gen = make_workload(npts=npts, seed_offset=rank)
    t0 = time.time()
    grid = H.Grid(hg, device=local, flags=H.BUILD_FP32)
    t_upload = time.time() - t0
    info = grid.info
    x = torch.from_numpy(X).to(dev)
    out32 = torch.empty((npts, TD), dtype=torch.float64, device=dev)
    out64 = torch.empty((npts, TD), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    def timed(plan, steps, warmup):
        """Replays of the plan's CUDA graph (autotuned node chunks)."""
        for _ in range(warmup):
            plan.launch(stream=stream)
        barrier()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
        ev[0].record(stream)
        for s in range(steps):
            plan.launch(stream=stream)
            ev[s + 1].record(stream)
        barrier()
        per = [ev[s].elapsed_time(ev[s + 1]) for s in range(steps)]
        total = ev[0].elapsed_time(ev[steps])
        return total, per, plan.launches

    if args.profile_replay:
        # two FP32C forward calls (a warm-up and a measured one) with a fixed
        # node-chunk size and kernel variant, nothing else: the case a
        # launch-level capture looks at (skip the first call's launches)
        chunk = args.chunk_rows if args.chunk_rows >= 0 else 64768
        H.set_chunk_rows(chunk)
        H.set_fp32c_variant(args.variant)
        for _ in range(2):
            H.interpolate(grid, x, precision=H.FP32C, out=out32, stream=stream)
        torch.cuda.synchronize(dev)
        print(json.dumps({"profile_replay": {"chunk_rows": chunk, "variant": args.variant,
                                             "launches_per_call": H.last_launch().kernels}}))
        return
    # accuracy of the FP32C form against the FP64 form (bit-identical to gold), all points
    H.interpolate(grid, x, precision=H.FP64, out=out64, stream=stream)
    H.interpolate(grid, x, precision=H.FP32C, out=out32, stream=stream)
    torch.cuda.synchronize(dev)
    den = torch.maximum(out64.abs(), 1e-3 * out64.abs().amax(dim=1, keepdim=True))
    perr = ((out32 - out64).abs() / den).amax(dim=1)
    err_max, err_rms = float(perr.max()), float(perr.pow(2).mean().sqrt())
    if args.only_accuracy_pass:
        H.active_count(grid, x, stream=stream)
        torch.cuda.synchronize(dev)
        print(json.dumps({"fp32c_max_rel_err": err_max, "fp32c_rms_rel_err": err_rms, "points": npts}))
        return
    # the tree walk alone (hit counting, no accumulation) over every point
    for _ in range(2):
        counts = H.active_count(grid, x, stream=stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    counts = H.active_count(grid, x, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    walk_ms = e0.elapsed_time(e1)
    mean_active = float(counts.double().mean())

    t_tune = time.time()
    plan32 = H.Plan(grid, x, out32, precision=H.FP32C, chunk_rows=args.chunk_rows, stream=stream)
    plan64 = H.Plan(grid, x, out64, precision=H.FP64, chunk_rows=args.chunk_rows, stream=stream)
    t_tune = time.time() - t_tune
    with Clocks(local) as clk:
        t32, per32, k32 = timed(plan32, args.steps, args.warmup)
        t64, per64, k64 = timed(plan64, args.steps, args.warmup)
    clocks = clk.summary()

    # end to end through the C ABI's host-pointer entry: pinned x in, pinned out back
    xh = torch.from_numpy(X).pin_memory()
    outh = torch.empty((npts, TD), dtype=torch.float64).pin_memory()
    import ctypes
    offs = np.array([0, npts], np.int64)
    garr = (ctypes.c_void_p * 1)(grid.handle.value)

    def e2e_once():
        rc = H.lib.sgi_interpolate_host(1, garr, offs.ctypes.data, xh.data_ptr(), outh.data_ptr(), H.FP32C)
        if rc:
            raise H.SgiError(rc, H.lib.sgi_last_error().decode())

    for _ in range(max(1, args.warmup)):
        e2e_once()
    barrier()
    te = time.perf_counter()
    for _ in range(args.steps):
        e2e_once()
    barrier()
    t_e2e = (time.perf_counter() - te) * 1e3

    # max over ranks
    def maxr(v):
        if world == 1:
            return v
        t = torch.tensor([v], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    t32, t64, t_e2e = maxr(t32), maxr(t64), maxr(t_e2e)
    result = None
    if rank == 0:
        hbm, peak_kind = peaks()
        b32, szxps = alg_bytes(hg, info, npts, 4)
        b64, _ = alg_bytes(hg, info, npts, 8)
        ms32 = t32 / args.steps
        ms64 = t64 / args.steps
        ach = b32 / (ms32 * 1e-3) / 1e9
        pts_s = npts * world / (ms32 * 1e-3)
        pts64_s = npts * world / (ms64 * 1e-3)
        traffic = FP32C_STEP_DRAM_BYTES if npts == NPTS else None
        result = {
            "metric": METRIC,
            "value": pts_s,
            "unit": "points/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms32,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32+comp (f64 in/out)",
            "data": "synthetic: seeded adaptive grid and points (reference's large grids are not in its tree)",
            "config": {"workload": WORKLOAD, "dim": DIM, "nno": info.nno, "TotalDof": TD, "points_per_gpu": npts,
                       "max_comps": info.max_comps, "ncoarse": info.ncoarse, "szxps": szxps,
                       "mean_active_nodes_per_point": mean_active,
                       "l2": "inputs larger than L2 (x 472 MB, surplus 1 GB FP32 / 2 GB FP64)",
                       "parallelism": f"replicated grid, points sharded, {world} GPU(s)"},
            "points_x_outputs_per_s": pts_s * TD,
            "fp64_form": {"points_per_s": pts64_s, "ms_per_step": ms64,
                          "roofline_frac": b64 / (ms64 * 1e-3) / 1e9 / hbm},
            "speedup_fp32c_vs_fp64_form": pts_s / pts64_s,
            "fp32c_vs_gold_exact_fp64": {"max_rel_err": err_max, "rms_rel_err": err_rms, "points": npts},
            "roofline": {"bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                         "peak_kind": f"{peak_kind} (burst copy)", "algorithmic_bytes_per_launch": b32,
                         "traffic": traffic, "kernel": "fwd_f32d_kernel",
                         "traffic_note": "ncu DRAM read+write of one forward call with node chunks of 64,768 "
                                         "(16 launches); the timed plan's chunking is in plans.fp32c"},
            "gather_roofline": gather_roof(mean_active, ms32, grid, hg),
            "walk_only_ms": walk_ms,
            "fma_work": {"mean_active_nodes": mean_active,
                         "flops_per_launch": 2.0 * mean_active * TD * npts,
                         "achieved_tflops": 2.0 * mean_active * TD * npts / (ms32 * 1e-3) / 1e12},
            "e2e": {"value": npts * world / (t_e2e / args.steps * 1e-3), "unit": "points/s",
                    "h2d_bytes_per_step": npts * DIM * 8, "d2h_bytes_per_step": npts * TD * 8},
            "gpu_launches": args.steps * (k32 + k64),
            "clocks": clocks,
            "setup_s": {"generate": round(t_gen, 2), "layout_and_upload": round(t_upload, 2),
                        "autotune_and_capture": round(t_tune, 2)},
            "plans": {"fp32c": {"chunk_rows": plan32.chunk_rows, "variant": plan32.variant,
                                "launches": plan32.launches},
                      "fp64": {"chunk_rows": plan64.chunk_rows, "launches": plan64.launches},
                      "note": "each step replays one CUDA graph holding all node-chunk launches"},
        }
    if rank == 0 and not args.no_cpu_baseline:
        result["cpu_baseline"] = cpu_baseline(hg, X, args.cpu_sample, args.cpu_variant)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(result))


def cpu_baseline(hg, X, sample, variant):
    """The reference's own CPU kernel (oracle/_ref) on a bounded sample of the
    workload's points, one call per point, all host threads."""
    import oracle as O
    if not O.ref_available(variant):
        return {"value": None, "unit": "points/s", "kind": "reference", "cores": 0,
                "sample": f"oracle/_ref/libref_{variant}.so not built"}
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "grid.plt")
        hg.write_plt(p)
        t = time.time()
        r = O.RefGrid(p, DIM, variant)
        t_load = time.time() - t
        cores = os.cpu_count() or 1
        half = len(X) // 2
        sub = np.ascontiguousarray(np.concatenate([X[:sample // 2], X[half:half + sample - sample // 2]]))
        r.interpolate(sub[:cores], nthreads=cores)
        t = time.perf_counter()
        r.interpolate(sub, nthreads=cores)
        dt = time.perf_counter() - t
    return {"value": len(sub) / dt, "unit": "points/s", "kind": "reference", "cores": cores,
            "variant": variant, "load_s": round(t_load, 1),
            "sample": f"{len(sub)} of the workload's points (half uniform, half clustered), "
                      f"LinearBasis_{variant}_Generic_InterpolateArray per point, {cores} threads"}


def run_reference(args):
    rank, world, _ = env_rank()
    if rank != 0:
        return
    import oracle as O
    variant = args.cpu_variant
    if not O.ref_available(variant):
        print(json.dumps({"impl": "reference", "unavailable": f"oracle/_ref/libref_{variant}.so not built "
                          "(needs the reference tree at build time)"}))
        return
    hg, X, _ = make_workload()
    cores = os.cpu_count() or 1
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "grid.plt")
        hg.write_plt(p)
        r = O.RefGrid(p, DIM, variant)
        rng = np.random.default_rng(0)
        times = []
        for s in range(args.warmup + args.steps):
            sub = X[rng.choice(NPTS, args.cpu_sample, replace=False)]
            t = time.perf_counter()
            r.interpolate(sub, nthreads=cores)
            if s >= args.warmup:
                times.append(time.perf_counter() - t)
    ms = float(np.mean(times)) * 1e3
    v = args.cpu_sample / (ms * 1e-3)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "points/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (same grid and points)",
        "config": {"workload": WORKLOAD, "sample_points_per_step": args.cpu_sample},
        "cpu_baseline": {"value": v, "unit": "points/s", "kind": "reference", "cores": cores,
                         "sample": f"{args.cpu_sample} random points of the workload per step, "
                                   f"LinearBasis_{variant}_Generic_InterpolateArray, {cores} threads"},
        "e2e": {"value": v, "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def _plan_time(H, torch, plan, stream, steps, warmup):
    for _ in range(warmup):
        plan.launch(stream=stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        plan.launch(stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def _rel_err(torch, a, b):
    den = torch.maximum(b.abs(), 1e-3 * b.abs().amax(dim=1, keepdim=True))
    e = ((a - b).abs() / den).amax(dim=1)
    return float(e.max()), float(e.pow(2).mean().sqrt())


def run_c2(args):
    """8 multistate grids (d=30, nno log-uniform in [20k, 200k], TotalDof=64), ragged
    batches of 1..100k uniform points per grid, one persistent launch per call."""
    import torch
    import hddm_b200 as H
    dev = torch.device("cuda", 0)
    rng = np.random.Generator(np.random.PCG64(2))
    nnos = np.exp(rng.uniform(np.log(20_000), np.log(200_000), 8)).astype(int)
    counts = rng.integers(1, 100_001, 8)
    hosts = [H.HostGrid.adaptive(30, int(n), 64, seed=200 + k) for k, n in enumerate(nnos)]
    grids = [H.Grid(h, flags=H.BUILD_FP32) for h in hosts]
    X = H.gen_points(30, int(counts.sum()), kind=0, seed=2)
    x = torch.from_numpy(X).to(dev)
    stream = torch.cuda.current_stream(dev)
    o32 = torch.empty((x.shape[0], 64), dtype=torch.float64, device=dev)
    o64 = torch.empty_like(o32)
    p32 = H.Plan(grids, x, o32, counts=list(counts), precision=H.FP32C, stream=stream)
    p64 = H.Plan(grids, x, o64, counts=list(counts), precision=H.FP64, stream=stream)
    ms32 = _plan_time(H, torch, p32, stream, args.steps, args.warmup)
    ms64 = _plan_time(H, torch, p64, stream, args.steps, args.warmup)
    emax, erms = _rel_err(torch, o32, o64)
    npts = int(counts.sum())
    print(json.dumps({"workload": "C2: 8 multistate grids d=30, TotalDof=64, ragged batches", "grids_nno": nnos.tolist(),
                      "points_per_grid": counts.tolist(), "points": npts,
                      "fp32c": {"ms": ms32, "points_per_s": npts / ms32 * 1e3, "variant": p32.variant,
                                "chunk_rows": p32.chunk_rows, "launches": p32.launches},
                      "fp64": {"ms": ms64, "points_per_s": npts / ms64 * 1e3, "launches": p64.launches},
                      "fp32c_vs_gold_exact_fp64": {"max_rel_err": emax, "rms_rel_err": erms}}))


def run_chunksweep(args):
    """Step time of both forms over fixed node-chunk sizes (the autotuner's
    search space, printed), default workload."""
    import torch
    import hddm_b200 as H
    dev = torch.device("cuda", 0)
    hg, X, _ = make_workload(npts=args.points)
    g = H.Grid(hg, flags=H.BUILD_FP32)
    x = torch.from_numpy(X).to(dev)
    out = torch.empty((X.shape[0], TD), dtype=torch.float64, device=dev)
    s = torch.cuda.current_stream(dev)
    rows_list = [0, 16384, 32768, 49152, 65536, 98304, 131072, 196608, 262144]
    res = {}
    for prec, name in ((H.FP32C, "fp32c"), (H.FP64, "fp64")):
        for rows in rows_list:
            p = H.Plan(g, x, out, precision=prec, chunk_rows=rows, stream=s)
            res.setdefault(name, []).append({"chunk_rows": rows, "launches": p.launches,
                                             "ms": _plan_time(H, torch, p, s, 3, 2)})
            del p
    print(json.dumps({"workload": WORKLOAD, "chunk_sweep": res}))


def run_variantsweep(args):
    """FP32C step time of every kernel variant over node-chunk sizes (direct
    calls, CUDA events), with each variant's error against the gold-exact FP64
    form, default workload."""
    import torch
    import hddm_b200 as H
    dev = torch.device("cuda", 0)
    hg, X, _ = make_workload(npts=args.points)
    g = H.Grid(hg, flags=H.BUILD_FP32)
    x = torch.from_numpy(X).to(dev)
    ref = H.interpolate(g, x, precision=H.FP64)
    rows_list = [int(r) for r in args.sweep_rows.split(",")]
    res = []
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for v in [int(k) for k in args.sweep_variants.split(",")]:
        H.set_fp32c_variant(v)
        for rows in rows_list:
            H.set_chunk_rows(rows)
            out = H.interpolate(g, x, precision=H.FP32C)
            torch.cuda.synchronize()
            e0.record()
            for _ in range(3):
                H.interpolate(g, x, precision=H.FP32C, out=out)
            e1.record()
            torch.cuda.synchronize()
            emax, erms = _rel_err(torch, out, ref)
            res.append({"variant": v, "chunk_rows": rows, "ms": e0.elapsed_time(e1) / 3,
                        "max_rel_err": emax, "rms_rel_err": erms})
            print(json.dumps(res[-1]), file=sys.stderr)
    H.set_fp32c_variant(-1)
    H.set_chunk_rows(-1)
    print(json.dumps({"workload": WORKLOAD, "variant_sweep": res}))


def run_c3(args):
    """Backward: d=59 adaptive grid of 300k nodes, TotalDof=128, 32768 points kept 1e-6
    from every kink; dL/dx and dL/dsurplus of L = sum c * f with c ~ N(0,1)."""
    import torch
    import hddm_b200 as H
    dev = torch.device("cuda", 0)
    hg = H.HostGrid.adaptive(59, 300_000, 128, seed=3)
    g = H.Grid(hg)
    X = H.gen_points(59, 32768, kind=0, seed=3, kink_reject=1e-6)
    C = np.random.Generator(np.random.PCG64(3)).standard_normal((32768, 128))
    x = torch.from_numpy(X).to(dev)
    c = torch.from_numpy(C).to(dev)
    for _ in range(args.warmup):
        H.backward(g, x, c)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        gx, gs = H.backward(g, x, c)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    e0.record()
    for _ in range(args.steps):
        H.interpolate(g, x)
    e1.record()
    torch.cuda.synchronize()
    fms = e0.elapsed_time(e1) / args.steps
    pairs = float(H.active_count(g, x).double().sum())
    print(json.dumps({"workload": "C3: backward, d=59, 300k nodes, TotalDof=128, 32768 points",
                      "backward_ms": ms, "forward_fp64_ms": fms, "active_pairs": pairs,
                      "backward_points_per_s": 32768 / ms * 1e3,
                      "grad_norms": {"dx": float(gx.norm()), "dsurplus": float(gs.norm())}}))


def run_errors(args):
    """FP32C max / RMS relative error against the FP64 form (bit-identical to the
    reference's gold path, as the GPU tests check), and both forms' step times
    (graph-plan replays), on every config's inputs:
    C0 regular d=4 level 4, TotalDof 8, 1024 points; C1 regular d=16 level 5,
    TotalDof 32, 65,536 points; C2 eight adaptive d=30 grids, TotalDof 64,
    ragged batches; C3 adaptive d=59, 300k nodes, TotalDof 128, 32,768
    points; C4 the benchmark workload."""
    import torch
    import hddm_b200 as H
    dev = torch.device("cuda", 0)

    stream = torch.cuda.current_stream(dev)

    def errs(grids, X, counts=None):
        x = torch.from_numpy(X).to(dev)
        o64 = H.interpolate(grids, x, counts=counts, precision=H.FP64)
        o32 = H.interpolate(grids, x, counts=counts, precision=H.FP32C)
        emax, erms = _rel_err(torch, o32, o64)
        # step times of autotuned graph plans of both forms (CUDA events)
        p64 = H.Plan(grids, x, o64, counts=counts, precision=H.FP64, stream=stream)
        p32 = H.Plan(grids, x, o32, counts=counts, precision=H.FP32C, stream=stream)
        ms64 = _plan_time(H, torch, p64, stream, max(args.steps, 5), args.warmup)
        ms32 = _plan_time(H, torch, p32, stream, max(args.steps, 5), args.warmup)
        return {"points": len(X), "max_rel_err": emax, "rms_rel_err": erms,
                "fp64_ms": ms64, "fp32c_ms": ms32, "fp32c_points_per_s": len(X) / ms32 * 1e3}

    res = {}
    g0 = H.HostGrid.regular(4, 4, 8, seed=0)
    res["C0"] = dict(nno=g0.nno, **errs(H.Grid(g0, flags=H.BUILD_FP32), H.gen_points(4, 1024, kind=0, seed=0)))
    g1 = H.HostGrid.regular(16, 5, 32, seed=1)
    res["C1"] = dict(nno=g1.nno, **errs(H.Grid(g1, flags=H.BUILD_FP32), H.gen_points(16, 65536, kind=0, seed=1)))
    rng = np.random.Generator(np.random.PCG64(2))
    nnos = np.exp(rng.uniform(np.log(20_000), np.log(200_000), 8)).astype(int)
    counts = rng.integers(1, 100_001, 8)
    grids = [H.Grid(H.HostGrid.adaptive(30, int(n), 64, seed=200 + k), flags=H.BUILD_FP32) for k, n in enumerate(nnos)]
    res["C2"] = dict(nno=nnos.tolist(), **errs(grids, H.gen_points(30, int(counts.sum()), kind=0, seed=2), list(counts)))
    del grids
    g3 = H.HostGrid.adaptive(59, 300_000, 128, seed=3)
    res["C3"] = dict(nno=g3.nno, **errs(H.Grid(g3, flags=H.BUILD_FP32),
                                         H.gen_points(59, 32768, kind=0, seed=3, kink_reject=1e-6)))
    hg, X, _ = make_workload()
    res["C4"] = dict(nno=hg.nno, **errs(H.Grid(hg, flags=H.BUILD_FP32), X))
    print(json.dumps({"fp32c_vs_gold_exact_fp64": res}))


def run_multistate(args):
    """The reference's own call shape: one point per state across 16 states
    (d=59, TotalDof=118, 200k nodes each), per-call latency."""
    import ctypes
    import torch
    import hddm_b200 as H
    dev = torch.device("cuda", 0)
    ns = 16
    hosts = [H.HostGrid.adaptive(59, 200_000, 118, seed=300 + k) for k in range(ns)]
    grids = [H.Grid(h, flags=H.BUILD_FP32) for h in hosts]
    X = H.gen_points(59, ns, kind=0, seed=5)
    arr = (ctypes.c_void_p * ns)(*[g.handle.value for g in grids])
    offs = np.arange(ns + 1, dtype=np.int64)
    xh = np.ascontiguousarray(X)
    outh = np.zeros((ns, 118))
    for _ in range(args.warmup):
        H.lib.sgi_interpolate_host(ns, arr, offs.ctypes.data, xh.ctypes.data, outh.ctypes.data, H.FP64)
    reps = max(args.steps, 50)
    t = time.perf_counter()
    for _ in range(reps):
        rc = H.lib.sgi_interpolate_host(ns, arr, offs.ctypes.data, xh.ctypes.data, outh.ctypes.data, H.FP64)
    host_s = (time.perf_counter() - t) / reps
    # one point on the first state, both forms
    single = {}
    off1 = np.array([0, 1], np.int64)
    for name, prec in (("fp64", H.FP64), ("fp32c", H.FP32C)):
        for _ in range(args.warmup):
            H.lib.sgi_interpolate_host(1, arr, off1.ctypes.data, xh.ctypes.data, outh.ctypes.data, prec)
        t = time.perf_counter()
        for _ in range(reps):
            H.lib.sgi_interpolate_host(1, arr, off1.ctypes.data, xh.ctypes.data, outh.ctypes.data, prec)
        single[name] = (time.perf_counter() - t) / reps
    x = torch.from_numpy(X).to(dev)
    out = torch.empty((ns, 118), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    plan = H.Plan(grids, x, out, counts=[1] * ns, precision=H.FP64, chunk_rows=0, stream=stream)
    dev_ms = _plan_time(H, torch, plan, stream, reps, args.warmup)
    print(json.dumps({"workload": "multistate call: 16 states x 1 point, d=59, TotalDof=118, 200k nodes per state",
                      "rc": rc, "host_call_s": host_s, "host_s_per_state": host_s / ns,
                      "graph_replay_ms": dev_ms, "graph_s_per_state": dev_ms * 1e-3 / ns,
                      "single_point_host_call_s": single,
                      "reference_published_s_per_state": {"large, cuda (daint)": 2.754e-4,
                                                          "large, avx2 (daint)": 4.234e-3}}))


def run_cutoffsweep(args):
    """FP32C step time (graph replay) and error against the gold-exact FP64 form
    for surplus cutoffs of 2^-k of the largest |surplus|, default workload."""
    import torch
    import hddm_b200 as H
    dev = torch.device("cuda", 0)
    hg, X, _ = make_workload(npts=args.points)
    g = H.Grid(hg, flags=H.BUILD_FP32)
    x = torch.from_numpy(X).to(dev)
    ref = H.interpolate(g, x, precision=H.FP64)
    smax = g.set_surplus_cutoff(0.0) * 2.0 ** 46
    stream = torch.cuda.Stream(dev)
    res = []
    for k in [int(v) for v in args.sweep_cutoffs.split(",")]:
        eff = g.set_surplus_cutoff(smax * 2.0 ** -k)
        out = torch.empty(x.shape[0], TD, dtype=torch.float64, device=dev)
        plan = H.Plan(g, x, out, precision=H.FP32C, chunk_rows=args.chunk_rows, stream=stream)
        ms = _plan_time(H, torch, plan, stream, 5, 3)
        emax, erms = _rel_err(torch, out, ref)
        res.append({"cutoff_log2_of_max_surplus": -k, "cutoff": eff, "ms": ms, "max_rel_err": emax,
                    "rms_rel_err": erms, "chunk_rows": plan.chunk_rows, "variant": plan.variant})
        print(json.dumps(res[-1]), file=sys.stderr)
        del plan
    g.set_surplus_cutoff(0.0)
    print(json.dumps({"workload": WORKLOAD, "cutoff_sweep": res}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="c4", choices=["c4", "c2", "c3", "multistate", "chunksweep", "variantsweep", "errors",
                                                        "cutoffsweep"],
                    help="c4 (default) is the benchmark line; the others print their own measurements")
    ap.add_argument("--cpu-sample", type=int, default=256)
    ap.add_argument("--sweep-variants", default="0,1,2", help="variantsweep: FP32C variants")
    ap.add_argument("--sweep-rows", default="0,131072,196608,262144,393216", help="variantsweep: chunk sizes")
    ap.add_argument("--sweep-cutoffs", default="46,40,36,34,32,30",
                    help="cutoffsweep: k of the cutoffs 2^-k * max|surplus| (46 is the default bound)")
    ap.add_argument("--cpu-variant", default="avx2", choices=["gold", "x86", "avx2"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--points", type=int, default=NPTS, help="points per GPU (default: the workload's 1M)")
    ap.add_argument("--chunk-rows", type=int, default=-1, help="node-chunk size of the plans (-1: autotune)")
    ap.add_argument("--variant", type=int, default=1, help="--profile-replay: FP32C kernel variant")
    ap.add_argument("--profile-replay", action="store_true",
                    help="only run two replays of the FP32C plan (launch-level profiling case)")
    ap.add_argument("--only-accuracy-pass", action="store_true",
                    help="run one FP64 and one FP32C launch, print their agreement and exit (profiling case)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "errors":
        run_errors(args)
    elif args.workload == "c2":
        run_c2(args)
    elif args.workload == "c3":
        run_c3(args)
    elif args.workload == "multistate":
        run_multistate(args)
    elif args.workload == "chunksweep":
        run_chunksweep(args)
    elif args.workload == "variantsweep":
        run_variantsweep(args)
    elif args.workload == "cutoffsweep":
        run_cutoffsweep(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
