"""Benchmark of the sparse-grid interpolation hot path on B200.

Workload (per GPU): one adaptive d=59 grid of 1,000,000 nodes grown by seeded
random refinement (levels <= 7), TotalDof = 256, and 1,000,000 query points
(first half uniform in [0,1]^59, second half N(0.5, 0.05^2) clipped to [0,1]).
A step is one forward pass over all points.  The headline form is the batched
FP32 + compensated kernel (SGI_FP32C); the plain FP64 kernel (bit-identical to
the reference's gold path) is timed beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

With N > 1 the benchmark runs one process per GPU: under torchrun (RANK /
WORLD_SIZE set) it is one of them; started directly it launches torchrun
itself.  Every rank replicates the grid and evaluates its own 1M points (weak
scaling, no collective on the data path; NCCL carries only the barrier and the
max-over-ranks timing).  `--impl reference` times the reference's own CPU code
(oracle/_ref, compiled from the reference sources) on the host cores over a
bounded sample of points per step, building its grid file and points with the
oracle's generator so that the product library is never loaded.
"""
import argparse
import json
import os
import socket
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "hddm-solver-postprocessors_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

DIM, NNO, TD, NPTS = 59, 1_000_000, 256, 1_000_000
GRID_SEED, POINT_SEED = 4, 40
CHECK_POINTS, CHECK_SEED = 4096, 40
METRIC = "d=59 points/s: batched FP32+comp vs plain FP64 GPU @<=1e-7 rel err; %HBM peak"
WORKLOAD = "C4: d=59 adaptive grid, 1M nodes (levels<=7), TotalDof=256, 1M points (half U[0,1], half N(0.5,0.05^2))"


def workload_config(npts=NPTS):
    """The workload as both arms name it (the reference arm times a sample of
    these points per step and says so in its cpu_baseline)."""
    return {"workload": WORKLOAD, "dim": DIM, "nno": NNO, "TotalDof": TD, "points_per_gpu": npts,
            "grid_seed": GRID_SEED, "point_seed": POINT_SEED,
            "l2": "inputs larger than L2 (x 472 MB, surplus rows 1 GB FP32 / 2 GB FP64)"}

# Random 1 KB surplus-row gathers from an L2-resident region (48 MB) with
# 16-byte loads, row indices read 32 at a time, measured on this pool's B200s
# by a standalone probe: 19.7-20.1 TB/s at 24 to 64 warps per SM and one to
# eight rows in flight per warp (20.2 TB/s for 512-byte rows).
GATHER_PEAK_TBS = 20.1
# Warps per SM of the FP32C kernel variants (blocks per SM x 8 warps).
VARIANT_WARPS = {0: 24, 1: 32, 2: 16}

# DRAM bytes (read + write) of one FP32C forward call of the default workload,
# keyed by node-chunk rows: the sum over one call's fwd_f32d_kernel launches
# in ncu captures of that chunking on 65,536 and 131,072 points (the bench's
# timed graph replay, --steps 1 --warmup 3), fitted as a + b * points (rows
# filled into the L2 once per chunk do not grow with the points; carried
# outputs, coordinates and row misses do), with the kernel variant the
# captures' plans chose.
FP32C_CALL_DRAM_BYTES = {97152: {"a": 4.016e8, "b": 60956.0, "variant": "2 at 65,536 points, 1 at 131,072"},
                         129536: {"a": 2.133e8, "b": 85875.0, "variant": "2 at 65,536 points, 1 at 131,072"}}


def env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def check_subsample():
    """The fixed 4,096-point subsample (seed 40) the oracle checks."""
    return np.sort(np.random.Generator(np.random.PCG64(CHECK_SEED)).choice(NPTS, CHECK_POINTS, replace=False))


def make_workload(npts=NPTS, seed_offset=0):
    import hddm_b200 as H
    t = time.time()
    hg = H.HostGrid.adaptive(DIM, NNO, TD, seed=GRID_SEED)
    X = H.gen_points(DIM, npts, kind=2, seed=POINT_SEED + seed_offset)
    return hg, X, time.time() - t


def alg_bytes(hg, info, npts, fp32c):
    """Algorithmic bytes of one forward call, each grid array counted once:
    coordinates and outputs (FP64) per point, the surplus rows (FP32 for FP32C,
    FP64 for the FP64 form), for FP32C also the FP64 copies of the coarse rows
    and the FP16 rows, chains (2 B per node per non-constant dimension) and
    unique xps (4 B)."""
    idx, _ = hg.arrays()
    i = idx[:, :DIM]
    j = idx[:, DIM:]
    nz = (i != 0) | (j != 0)
    dims = np.broadcast_to(np.arange(DIM), i.shape)[nz].astype(np.int64)
    keys = (dims << 32) | (i[nz].astype(np.int64) << 16) | j[nz].astype(np.int64)
    szxps = int(np.unique(keys).size) + 1
    rows = info.nno * TD * 4 + info.ncoarse * TD * 8 + info.nno * TD * 2 if fp32c else info.nno * TD * 8
    return npts * DIM * 8 + npts * TD * 8 + rows + 2 * info.nno * info.max_comps + 4 * szxps, szxps


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


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def spawn_ranks(n):
    """One process per GPU: re-run this command under torchrun with n ranks."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", f"--master-port={free_port()}", os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def init_ranks(args, backend):
    """Process group of the launched ranks; WORLD_SIZE must equal --gpus."""
    import datetime
    import torch.distributed as dist
    rank, world, local = env_rank()
    if world != args.gpus:
        raise SystemExit(f"--gpus {args.gpus} but WORLD_SIZE={world}")
    if world > 1:
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return rank, world, local


def max_over_ranks(values, world, device):
    import torch
    import torch.distributed as dist
    if world == 1:
        return list(values)
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]


def run_launch_check(args):
    """The launcher, process group, barrier and max-over-ranks reduction of the
    multi-GPU path on CPU (gloo), without any GPU work: every rank reports a
    time of rank + 1 ms and rank 0 prints the maximum."""
    import torch.distributed as dist
    rank, world, _ = init_ranks(args, "gloo")
    if world > 1:
        dist.barrier()
    (ms,) = max_over_ranks([rank + 1.0], world, "cpu")
    if rank == 0:
        print(json.dumps({"launch_check": "ok", "n_gpus": world, "max_over_ranks_ms": ms}))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_gpu(args):
    import ctypes
    import torch
    import torch.distributed as dist

    import hddm_b200 as H

    rank, world, local = init_ranks(args, "nccl")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
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
        """Replays of the plan's CUDA graph; CUDA events on the replay stream."""
        for _ in range(warmup):
            plan.launch(stream=stream)
        barrier()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
        ev[0].record(stream)
        for s in range(steps):
            plan.launch(stream=stream)
            ev[s + 1].record(stream)
        barrier()
        return ev[0].elapsed_time(ev[steps])

    t_tune = time.time()
    plan32 = H.Plan(grid, x, out32, precision=H.FP32C, chunk_rows=args.chunk_rows, stream=stream)
    plan64 = H.Plan(grid, x, out64, precision=H.FP64, chunk_rows=args.chunk_rows, stream=stream)
    t_tune = time.time() - t_tune
    with Clocks(local) as clk:
        t32 = timed(plan32, args.steps, args.warmup)
        t64 = timed(plan64, args.steps, args.warmup)
    clocks = clk.summary()

    # end to end through the C ABI's host-pointer entry: pinned x in, pinned out back
    xh = torch.from_numpy(X).pin_memory()
    outh = torch.empty((npts, TD), dtype=torch.float64).pin_memory()
    offs = np.array([0, npts], np.int64)
    garr = (ctypes.c_void_p * 1)(grid.handle.value)

    def e2e_once():
        rc = H.lib.sgi_interpolate_host(1, garr, offs.ctypes.data, xh.data_ptr(), outh.data_ptr(), H.FP32C)
        if rc:
            raise H.SgiError(rc, H.lib.sgi_last_error().decode())

    for _ in range(args.warmup):
        e2e_once()
    barrier()
    te = time.perf_counter()
    for _ in range(args.steps):
        e2e_once()
    barrier()
    t_e2e = (time.perf_counter() - te) * 1e3

    # untimed: the walk alone, and the terms per class (the bytes the FP32C
    # kernels gather), over every point
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    H.active_count(grid, x, stream=stream)
    e0.record(stream)
    counts = H.active_count(grid, x, stream=stream)
    e1.record(stream)
    classes = H.term_classes(grid, x, stream=stream).sum(dim=0)
    torch.cuda.synchronize(dev)
    walk_ms = e0.elapsed_time(e1)
    pairs = float(counts.double().sum())
    n_big, n_fine, n_half, n_drop = (float(v) for v in classes.cpu())
    o64_sub = o32_sub = None
    if world == 1 and npts == NPTS:
        sub = torch.from_numpy(check_subsample()).to(dev)
        o64_sub = out64.index_select(0, sub).cpu().numpy()
        o32_sub = out32.index_select(0, sub).cpu().numpy()

    t32, t64, t_e2e = max_over_ranks([t32, t64, t_e2e], world, dev)
    result = None
    if rank == 0:
        hbm, peak_kind = peaks()
        b32, szxps = alg_bytes(hg, info, npts, True)
        ms32 = t32 / args.steps
        ms64 = t64 / args.steps
        b64, _ = alg_bytes(hg, info, npts, False)
        pts_s = npts * world / (ms32 * 1e-3)
        pts64_s = npts * world / (ms64 * 1e-3)
        ach = b32 / (ms32 * 1e-3) / 1e9
        gather_b = n_fine * info.ld * 4 + n_half * info.ld * 2 + n_big * info.ld * 8
        warps = VARIANT_WARPS.get(plan32.variant % 3, 32)
        gpeak = GATHER_PEAK_TBS
        gach = gather_b / (ms32 * 1e-3) / 1e12
        sm_mhz = clocks.get("sm_mhz") or 1965.0
        fp32_peak = 148 * 128 * 2 * sm_mhz * 1e6 / 1e12
        flops = 2.0 * pairs * TD
        tfit = FP32C_CALL_DRAM_BYTES.get(plan32.chunk_rows)
        traffic = tfit["a"] + tfit["b"] * npts if tfit else None
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
            "data": "synthetic: seeded adaptive grid and points (the reference's large grids are not in its tree)",
            "config": workload_config(npts),
            "parallelism": f"replicated grid, points sharded, {world} GPU(s)",
            "workload_stats": {"nno": info.nno, "max_comps": info.max_comps, "ncoarse": info.ncoarse,
                               "szxps": szxps, "mean_active_nodes_per_point": pairs / npts},
            "points_x_outputs_per_s": pts_s * TD,
            "fp64_form": {"points_per_s": pts64_s, "ms_per_step": ms64,
                          "roofline_frac": b64 / (ms64 * 1e-3) / 1e9 / hbm},
            "speedup_fp32c_vs_fp64_form": pts_s / pts64_s,
            "roofline": {"bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                         "traffic": traffic, "peak_kind": f"{peak_kind} (burst copy)",
                         "algorithmic_bytes_per_call": b32, "kernel": "fwd_f32d_kernel",
                         "per": f"one forward call: one CUDA-graph replay of {plan32.launches} node-chunk launches",
                         "traffic_note": "ncu DRAM read+write of one call with the plan's chunking, fitted "
                                         "over 65,536 and 131,072 points and taken at this run's points "
                                         "(null when that chunking was not captured)",
                         "traffic_capture_variant": tfit["variant"] if tfit else None},
            "gather_roofline": {"bound": "l2_row_gather", "achieved": gach, "unit": "TB/s",
                                "peak": gpeak, "frac": gach / gpeak,
                                "bytes_per_call": gather_b, "kernel_warps_per_sm": warps,
                                "terms": {"big_fp64_rows": n_big, "fine_fp32_rows": n_fine,
                                          "fine_fp16_rows": n_half, "dropped": n_drop},
                                "note": "rows the FP32C kernel reads: fine terms x TotalDof x 4 B (FP32 rows) or "
                                        "x 2 B (FP16 rows) + big terms x TotalDof x 8 B (dropped terms read none), "
                                        "over the step time; peak: random 1 KB row gathers from an L2-resident "
                                        "region (standalone probe)"},
            "fma_work": {"active_pairs_per_call": pairs, "flops_per_call": flops,
                         "achieved_tflops": flops / (ms32 * 1e-3) / 1e12,
                         "fp32_peak_tflops": fp32_peak, "frac": flops / (ms32 * 1e-3) / 1e12 / fp32_peak,
                         "note": "2 x TotalDof per active (point, node) pair; peak: nominal 148 SMs x 128 FP32 "
                                 "lanes x 2 at the median SM clock sampled in the timed region"},
            "walk_only_ms": walk_ms,
            "e2e": {"value": npts * world / (t_e2e / args.steps * 1e-3), "unit": "points/s",
                    "h2d_bytes_per_step": npts * DIM * 8, "d2h_bytes_per_step": npts * TD * 8},
            "gpu_launches": args.steps * plan32.launches,
            "clocks": clocks,
            "setup_s": {"generate": round(t_gen, 2), "layout_and_upload": round(t_upload, 2),
                        "autotune_and_capture": round(t_tune, 2)},
            "plans": {"fp32c": {"chunk_rows": plan32.chunk_rows, "variant": plan32.variant,
                                "launches": plan32.launches},
                      "fp64": {"chunk_rows": plan64.chunk_rows, "launches": plan64.launches},
                      "note": "each step replays one CUDA graph holding all node-chunk launches; gpu_launches "
                              "counts the FP32C steps' kernels"},
        }
        if world == 1 and not args.no_cpu_baseline:
            result.update(cpu_leg(hg, X, o64_sub, o32_sub, args.cpu_sample))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(result))


def cpu_flags():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("flags"):
                return set(line.split(":", 1)[1].split())
    except OSError:
        pass
    return set()


def ref_variants():
    """The reference's SIMD CPU kernels built under oracle/_ref that this host
    can run and that agree with gold: avx2.  (The reference's avx512 kernel
    needs the Intel compiler's OpenMP reduction; built without it, it
    reproduces the reference's fixture but not gold on generated grids.)"""
    import oracle as O
    return ["avx2"] if O.ref_available("avx2") and {"avx2", "fma"} <= cpu_flags() else []


def cpu_leg(hg, X, o64_sub, o32_sub, sample):
    """Host-side leg (rank 0, one GPU): the oracle checks the timed plans'
    outputs on the 4,096-point subsample (FP64 bit for bit, FP32C relative
    error), and the reference's own SIMD CPU kernel (oracle/_ref, avx2) is
    timed on a bounded sample of the workload's points, one call per point,
    all host threads."""
    import oracle as O
    cores = os.cpu_count() or 1
    res = {}
    if o64_sub is not None:
        sub = check_subsample()
        ref = O.Gold(*hg.arrays()).interpolate(X[sub], nthreads=cores)
        emax, erms = O.rel_error(o32_sub, ref)
        res["parity_vs_oracle"] = {
            "points": CHECK_POINTS, "subsample_seed": CHECK_SEED,
            "fp64_bit_exact_vs_oracle": bool(np.array_equal(o64_sub, ref)),
            "fp64_max_abs_diff": float(np.abs(o64_sub - ref).max()),
            "fp32c_vs_oracle_gold": {"max_rel_err": emax, "rms_rel_err": erms},
            "note": "outputs of the last timed replay of each plan against the oracle's gold restatement"}
    variants = ref_variants()
    if not variants:
        res["cpu_baseline"] = {"value": None, "unit": "points/s", "kind": "reference", "cores": 0,
                               "sample": "no reference SIMD kernel under oracle/_ref that this host can run"}
        return res
    half = len(X) // 2
    pts = np.ascontiguousarray(np.concatenate([X[:sample // 2], X[half:half + sample - sample // 2]]))
    rates, loads = {}, {}
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "grid.plt")
        hg.write_plt(p)
        for variant in variants:
            t = time.time()
            r = O.RefGrid(p, DIM, variant)
            loads[variant] = round(time.time() - t, 1)
            r.interpolate(pts[:cores], nthreads=cores)
            t = time.perf_counter()
            r.interpolate(pts, nthreads=cores)
            rates[variant] = len(pts) / (time.perf_counter() - t)
            del r
    best = max(rates, key=rates.get)
    res["cpu_baseline"] = {"value": rates[best], "unit": "points/s", "kind": "reference", "cores": cores,
                           "variant": best, "points_per_s_by_variant": rates, "load_s": loads,
                           "sample": f"{len(pts)} of the workload's points (half uniform, half clustered), "
                                     f"LinearBasis_<variant>_Generic_InterpolateArray per point, {cores} threads"}
    return res


def run_reference(args):
    """The reference's own CPU kernel over a bounded sample of the workload per
    step; the grid file and the points come from the oracle's generator (the
    product library is not loaded)."""
    rank, world, _ = env_rank()
    if rank != 0:
        return
    import oracle as O
    variant = args.cpu_variant
    if variant == "auto":
        variant = "avx2"
    if not O.ref_available(variant):
        print(json.dumps({"impl": "reference", "unavailable": f"oracle/_ref/libref_{variant}.so not built "
                          "(needs the reference tree at build time)"}))
        return
    cores = os.cpu_count() or 1
    og = O.Gold.adaptive(DIM, NNO, TD, GRID_SEED)
    X = O.gen_points(DIM, NPTS, 2, POINT_SEED)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "grid.plt")
        og.write_plt(p)
        del og
        r = O.RefGrid(p, DIM, variant)
        rng = np.random.default_rng(0)
        times = []
        for s in range(args.warmup + args.steps):
            sub = X[rng.choice(NPTS, args.ref_sample, replace=False)]
            t = time.perf_counter()
            r.interpolate(sub, nthreads=cores)
            if s >= args.warmup:
                times.append(time.perf_counter() - t)
    ms = float(np.mean(times)) * 1e3
    v = args.ref_sample / (ms * 1e-3)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "points/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (same grid and points)",
        "config": workload_config(),
        "parallelism": f"host threads over points, {cores} threads",
        "cpu_baseline": {"value": v, "unit": "points/s", "kind": "reference", "cores": cores,
                         "sample": f"{args.ref_sample} random points of the workload per step, "
                                   f"LinearBasis_{variant}_Generic_InterpolateArray, {cores} threads"},
        "e2e": {"value": v, "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def _plan_time(torch, plan, stream, steps, warmup):
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
    ms32 = _plan_time(torch, p32, stream, args.steps, args.warmup)
    ms64 = _plan_time(torch, p64, stream, args.steps, args.warmup)
    npts = int(counts.sum())
    print(json.dumps({"workload": "C2: 8 multistate grids d=30, TotalDof=64, ragged batches", "grids_nno": nnos.tolist(),
                      "points_per_grid": counts.tolist(), "points": npts,
                      "fp32c": {"ms": ms32, "points_per_s": npts / ms32 * 1e3, "variant": p32.variant,
                                "chunk_rows": p32.chunk_rows, "launches": p32.launches},
                      "fp64": {"ms": ms64, "points_per_s": npts / ms64 * 1e3, "launches": p64.launches}}))


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
        H.backward(g, x, c)
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
    # bytes the backward must move at least: coordinates, dL/dvalue and dL/dx
    # per point, one FP64 surplus row read and one dL/dsurplus row written per node
    b_alg = 32768 * (59 * 8 * 2 + 128 * 8) + hg.nno * 128 * 8 * 2
    print(json.dumps({"workload": "C3: backward, d=59, 300k nodes, TotalDof=128, 32768 points",
                      "backward_ms": ms, "forward_fp64_ms": fms, "active_pairs": pairs,
                      "backward_points_per_s": 32768 / ms * 1e3,
                      "algorithmic_bytes": b_alg, "pair_row_bytes": pairs * 128 * 8 * 2,
                      "pair_row_tbs": pairs * 128 * 8 * 2 / (ms * 1e-3) / 1e12}))


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
    dev_ms = _plan_time(torch, plan, stream, reps, args.warmup)
    print(json.dumps({"workload": "multistate call: 16 states x 1 point, d=59, TotalDof=118, 200k nodes per state",
                      "rc": rc, "host_call_s": host_s, "host_s_per_state": host_s / ns,
                      "graph_replay_ms": dev_ms, "graph_s_per_state": dev_ms * 1e-3 / ns,
                      "single_point_host_call_s": single,
                      "reference_published_s_per_state": {"large, cuda (daint)": 2.754e-4,
                                                          "large, avx2 (daint)": 4.234e-3}}))


def run_load(args):
    """Grid load time of the benchmark grid (d=59, 1M nodes, TotalDof 256)
    from its .plt file: parse + layout build + upload, against a load through
    the layout cache (the file's cache written by a first load)."""
    import torch
    import hddm_b200 as H
    torch.cuda.init()
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "grid.plt")
        H.HostGrid.adaptive(DIM, NNO, TD, seed=GRID_SEED).write_plt(p)
        t = time.perf_counter()
        hg = H.HostGrid.read_plt(p, DIM)
        t_read = time.perf_counter() - t
        g = H.Grid(hg, flags=H.BUILD_FP32)
        t_build = time.perf_counter() - t
        del g, hg
        t = time.perf_counter()
        g = H.Grid.load(p, DIM, flags=H.BUILD_FP32)
        t_first = time.perf_counter() - t
        del g
        t = time.perf_counter()
        g = H.Grid.load(p, DIM, flags=H.BUILD_FP32)
        t_cached = time.perf_counter() - t
        hit = g.cache_hit
        sizes = {"plt_bytes": os.path.getsize(p), "cache_bytes": os.path.getsize(p + ".sgi-layout")}
    print(json.dumps({"workload": "grid load: d=59, 1M nodes, TotalDof 256, FP64 + FP32C forms",
                      "read_plt_s": t_read, "read_build_upload_s": t_build,
                      "first_load_with_cache_write_s": t_first, "cached_load_s": t_cached, "cache_hit": hit,
                      **sizes}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="c4", choices=["c4", "c2", "c3", "multistate", "load"],
                    help="c4 (default) is the benchmark line; the others print their own measurements")
    ap.add_argument("--cpu-sample", type=int, default=16384,
                    help="points of the CPU baseline's timed sample (default: 16,384)")
    ap.add_argument("--ref-sample", type=int, default=2048, help="--impl reference: points per step")
    ap.add_argument("--cpu-variant", default="auto", choices=["auto", "gold", "x86", "avx2"],
                    help="--impl reference: the reference CPU kernel (auto: avx2)")
    ap.add_argument("--no-cpu-baseline", action="store_true",
                    help="skip the host leg (oracle check of the outputs and the CPU baseline)")
    ap.add_argument("--points", type=int, default=NPTS, help="points per GPU (default: the workload's 1M)")
    ap.add_argument("--chunk-rows", type=int, default=-1, help="node-chunk size of the plans (-1: autotune)")
    ap.add_argument("--launch-check", action="store_true",
                    help="check the multi-rank launcher and the max-over-ranks reduction on CPU (gloo), no GPU work")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ and args.impl == "b200":
        sys.exit(spawn_ranks(args.gpus))
    if args.launch_check:
        run_launch_check(args)
    elif args.impl == "reference":
        run_reference(args)
    elif args.workload == "c2":
        run_c2(args)
    elif args.workload == "c3":
        run_c3(args)
    elif args.workload == "multistate":
        run_multistate(args)
    elif args.workload == "load":
        run_load(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
