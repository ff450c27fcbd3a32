#!/usr/bin/env python
"""Benchmark of the IB coupling operators (spread + interpolate) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload large-channel|medium-channel|channel|single-rbc]
                    [--precision fp32c|fp64] [--no-cpu] [--no-extras]
                    [--leg all|batched|serving|membrane|fluid]

One step = ibk_spread_interpolate over every Lagrangian point of the
workload: one spread and one interpolation at the same positions, which bin
the points once (spread overwrites all grid faces, interpolate writes every
point velocity).  Metric: points per second through spread+interp, in the chosen
FP32C form, with the plain FP64 path, its accuracy, p50/p99 step times, the
end-to-end rate through host buffers and the CPU baseline in the same line.

The same line also carries four legs (skipped with --no-extras, or run
alone with --leg): "batched" -- 256 independent instances (cube grids 32^3..128^3,
1-50 cells each) in graph-captured persistent launches (spread and
interpolation, one binning), FP32C against the FP64 batch and against a loop
of single plans; "serving" -- the
256 instances as device-resident members stepped (interpolate, advect, spring
force, spread) under Poisson request arrivals from 1k to 50k steps/s, with
p50/p99 latency per offered rate; "fluid" -- one implicit diffusion step of
a velocity component on the large channel's grid; "membrane" -- the producers of the point
forces, for 64 shapes of the reference's RBC discretisation (2500 data sites,
10000 samples): surface geometry (FP64 operator products, normals, patch
areas) and the Skalak tension, per step.

Default workload: the large channel, 128 x 64 x 128 um, MAC grid 512 x 256 x
512 (h = 0.25 um), 3300 RBCs x 2210 points + 6000 platelets x 605 points =
10,923,000 points, bspline<3> delta, forces / velocities iid N(0,1).  Its grid
fields (1.6 GB per field) are far larger than the 126 MB L2, so no flush is
needed between steps; smaller workloads flush L2 between timed steps.

Under torchrun (N > 1) every rank runs an independent replica of the workload
(the operators have no exchange step on one domain); value = points of all
ranks / max-over-ranks time.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "spread+interp points/s"
L2_BYTES = 126 * 1024 * 1024

# DRAM bytes moved by one launch of the dominant kernel per algorithmic byte,
# from one ncu capture (dram__bytes_read.sum + dram__bytes_write.sum) of the
# FP32C spread on the 256 x 128 x 256 channel (1,364,270 points): 230.18 MB
# against 266.29 MB (part of the written grid is still dirty in L2 when the
# kernel ends).  Points and faces both scale by 8.01 to the 512 x 256 x 512
# channel, so a launch's traffic is this ratio times its algorithmic bytes.
TRAFFIC_PER_ALGORITHMIC_BYTE = {("spread_tile_kernel", "fp32c"): 230.18e6 / 266.29e6}


def load_package():
    import importlib.util
    if "ib_cu_b200" in sys.modules:
        return sys.modules["ib_cu_b200"]
    pkg_dir = os.path.join(ROOT, "ib.cu_b200")
    spec = importlib.util.spec_from_file_location(
        "ib_cu_b200", os.path.join(pkg_dir, "__init__.py"), submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["ib_cu_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# --------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clock / throttle-reason samples while the timed loop runs."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200", "-f", self.path],
                stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if self.proc is None or not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------ workloads
def max_over_ranks(ms, world, device):
    """The job's time: the largest per-rank device time (all_reduce MAX)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def make_workload(name, seed=0):
    load_package()
    from ib_cu_b200 import workloads as W
    return W.CONFIGS[name](seed=seed)


def grid_faces(plan):
    return sum(plan.sizes())


def algorithmic_bytes(n_points, faces):
    """Per operator: read x and F (or write U): 48 B per point; write (spread)
    or read (interpolate) every face once: 8 B per face."""
    return 48 * n_points + 8 * faces


class CpuStep:
    """One full spread + interpolate of the workload through the oracle's
    multi-threaded restatement of the reference algorithm (every point, the
    full grid), timed on the host cores: the CPU baseline and the reference
    arm.  Nothing is sampled or scaled."""

    def __init__(self, w, threads=0):
        from oracle import oracle as O
        from ib_cu_b200 import workloads as W
        O.build()
        self.O, self.w = O, w
        self.g = O.geometry(w.dims, w.lengths, w.boundaries, O.TAG_MAC, w.refinement)
        # every host CPU this process may run on: torchrun sets OMP_NUM_THREADS=1
        # per rank, which the oracle's explicit thread count overrides
        self.threads = threads or max(len(os.sched_getaffinity(0)), O.max_threads())
        sizes = [int(self.g.size[c]) for c in range(w.dims)]
        rng = np.random.default_rng(w.seed + 1)
        self.ue = [rng.normal(size=s_) * W.UM_PER_S for s_ in sizes]
        self.fe = [np.zeros(s_) for s_ in sizes]

    def step(self):
        """Seconds of one full spread + interpolate."""
        O, w = self.O, self.w
        t0 = time.perf_counter()
        O.spread(self.g, w.x, w.f, fe=self.fe, threads=self.threads)
        O.interpolate(self.g, w.x, self.ue, threads=self.threads)
        return time.perf_counter() - t0

    def describe(self, steps):
        return (f"oracle spread+interp (reference algorithm, {self.threads} threads), the full workload "
                f"({self.w.n} points, full grid), {steps} whole step(s) timed, median")


def cpu_measure(w, threads=0):
    """CPU baseline of the main line: one whole oracle step of the workload."""
    cs = CpuStep(w, threads)
    t = cs.step()
    return {"value": w.n / t, "unit": "points/s", "cores": cs.threads, "kind": "port",
            "sample": cs.describe(1), "t_full_s": t}


# Whole reference steps take about half a minute on the host cores: the arm
# runs at most this many timed steps (and at most one warm-up step).
REFERENCE_MAX_STEPS = 3


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    w = make_workload(args.workload)
    cs = CpuStep(w)
    for _ in range(min(args.warmup, 1)):
        cs.step()
    steps = max(1, min(args.steps, REFERENCE_MAX_STEPS))
    times = [cs.step() for _ in range(steps)]
    t_full = statistics.median(times)
    v = w.n / t_full
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "points/s",
        "n_gpus": args.gpus, "steps": steps, "steps_requested": args.steps, "warmup": min(args.warmup, 1),
        "ms_per_step": 1000.0 * t_full,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": workload_config(w, "fp64"),
        "cpu_baseline": {"value": v, "unit": "points/s", "cores": cs.threads, "kind": "port",
                         "sample": cs.describe(steps)},
        "e2e": {"value": v, "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": (f"whole steps of the full workload, capped at {REFERENCE_MAX_STEPS} timed steps and one "
                 "warm-up (about half a minute each); the reference's GPU build does not compile with "
                 "nvcc 12.9 (device lambdas in private members, legacy cuSPARSE API), so this arm times "
                 "the oracle's multi-threaded restatement of the reference algorithm on the host cores"),
    }
    print(json.dumps(line), flush=True)


def workload_config(w, precision):
    return {"workload": w.name, "points": int(w.n),
            "grid": "x".join(str(int(round(l / 0.025))) for l in w.lengths),
            "boundaries": ["periodic" if b == 0 else "solid" for b in w.boundaries],
            "delta": "bspline<3>", "precision": precision,
            "l2": ("inputs larger than L2" if w.name.startswith(("large", "medium"))
                   else "L2 flushed between steps")}


# ----------------------------------------------------------- GPU arm
def run_ours(args):
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)
    ibk = load_package()
    ibk.lib()
    from ib_cu_b200 import workloads as W

    if args.leg in ("batched", "serving", "membrane", "fluid"):
        # one leg alone (profiling runs): its own JSON object
        if args.leg == "batched":
            res = run_batched(ibk, W, dev, seed=0, steps=max(5, args.steps), rank=rank, world=world)
        elif args.leg == "membrane":
            res = run_membrane(ibk, dev, steps=max(5, args.steps))
        elif args.leg == "fluid":
            res = run_fluid(ibk, W, dev, steps=max(3, args.steps // 2), workload=args.workload)
        else:
            res = run_serving(ibk, W, dev, seed=rank, rates=[1000, 2000, 5000, 10000, 20000, 50000])
        if rank == 0:
            print(json.dumps({"leg": args.leg, args.leg: res}), flush=True)
        return

    w = make_workload(args.workload, seed=rank)
    precision = {"fp64": ibk.FP64, "fp32c": ibk.FP32C}[args.precision]
    dom = ibk.Domain(*[ibk.Dimension(l, b) for l, b in zip(w.lengths, w.boundaries)])
    plan = ibk.Plan(ibk.Mac(w.refinement), dom, ibk.Bspline(3), precision)
    plan.reserve(w.n)
    n = w.n
    sizes = plan.sizes()
    G = sum(sizes)
    stream = torch.cuda.current_stream()
    gen = torch.Generator(device=dev)
    gen.manual_seed(1000 + rank)
    x = torch.from_numpy(w.x).to(dev)
    f = torch.from_numpy(w.f).to(dev)
    ue = [torch.randn(s, generator=gen, dtype=torch.float64, device=dev) * W.UM_PER_S for s in sizes]
    fe = [torch.empty(s, dtype=torch.float64, device=dev) for s in sizes]
    ul = torch.empty(3 * n, dtype=torch.float64, device=dev)
    big = (8 * G) > L2_BYTES
    flush = None if big else torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=dev)

    def step():
        # one spread and one interpolation at the same positions (one binning)
        plan.spread_interpolate(n, x, f, fe, ue, ul, stream)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(max(args.warmup, 3)):
        step()
    barrier()
    plan.check()

    # ---- timed region: device-resident inputs, CUDA events on the stream
    launches0 = plan.launch_count()
    with ClockSampler(local) as clk:
        barrier()
        if flush is None:
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(args.steps):
                step()
            e1.record(stream)
            torch.cuda.synchronize()
            elapsed = e0.elapsed_time(e1)
        else:
            elapsed = 0.0
            for _ in range(args.steps):
                flush.zero_()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                step()
                e1.record(stream)
                torch.cuda.synchronize()
                elapsed += e0.elapsed_time(e1)
        barrier()
    launches = plan.launch_count() - launches0
    ms_total = max_over_ranks(elapsed, world, dev)
    ms_step = ms_total / args.steps
    value = world * n / (ms_step / 1000.0)
    clocks = clk.summary()

    # ---- per-kernel device times (profiled pass, same steps) for the roofline
    plan.reset_stats()
    plan.set_profiling(True)
    for _ in range(args.steps):
        if flush is not None:
            flush.zero_()
        step()
    stats = plan.kernel_stats()
    plan.set_profiling(False)
    peak, peak_kind = measured_peaks()
    top = max(stats.items(), key=lambda kv: kv[1][1]) if stats else (None, (0, 0.0))
    name, (nl, tot) = top
    avg_ms = tot / max(nl, 1)
    op_bytes = algorithmic_bytes(n, G)
    achieved = op_bytes / (avg_ms / 1000.0) / 1e9 if avg_ms > 0 else 0.0
    ratio = TRAFFIC_PER_ALGORITHMIC_BYTE.get((name, args.precision))
    traffic = ratio * op_bytes if ratio is not None else None
    traffic_source = ("ncu dram bytes of the FP32C spread on the 256x128x256 channel, scaled by units "
                      "processed (x8.01)" if ratio is not None else None)
    kernels = {k: {"launches": v[0], "avg_ms": v[1] / max(v[0], 1),
                   "share": v[1] / max(sum(s[1] for s in stats.values()), 1e-12)}
               for k, v in stats.items()}

    # ---- end to end through the public API with pinned host buffers
    xh = torch.from_numpy(w.x).pin_memory()
    fh = torch.from_numpy(w.f).pin_memory()
    ulh = [torch.empty(3 * n, dtype=torch.float64).pin_memory() for _ in range(2)]

    def e2e_step():
        x.copy_(xh, non_blocking=True)
        f.copy_(fh, non_blocking=True)
        step()
        ulh[0].copy_(ul, non_blocking=True)

    # (a) serial: upload, compute, download, one step after the other
    for _ in range(2):
        e2e_step()
    barrier()
    e2e_serial_ms = 0.0
    for _ in range(args.steps):
        if flush is not None:
            flush.zero_()
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        e2e_step()
        a1.record(stream)
        torch.cuda.synchronize()
        e2e_serial_ms += a0.elapsed_time(a1)
    e2e_serial = world * n / (max_over_ranks(e2e_serial_ms, world, dev) / args.steps / 1000.0)

    # (b) pipelined: two input and two output buffers; step k's upload runs on
    # one copy stream while step k-1 computes, its download on another while
    # step k+1 computes.  Every step still uploads its x and F and downloads
    # its U inside the timed region.
    xs, fs_, uls = [x, torch.empty_like(x)], [f, torch.empty_like(f)], [ul, torch.empty_like(ul)]
    s_in, s_out = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    ev = {k: [torch.cuda.Event() for _ in range(2)] for k in ("in", "comp", "out")}

    def e2e_pipelined(k_steps):
        for i in range(k_steps):
            b = i % 2
            s_in.wait_event(ev["comp"][b])           # buffers b free once step i-2 computed
            with torch.cuda.stream(s_in):
                xs[b].copy_(xh, non_blocking=True)
                fs_[b].copy_(fh, non_blocking=True)
            ev["in"][b].record(s_in)
            stream.wait_event(ev["in"][b])
            stream.wait_event(ev["out"][b])          # U buffer b downloaded (step i-2)
            plan.spread_interpolate(n, xs[b], fs_[b], fe, ue, uls[b], stream)
            ev["comp"][b].record(stream)
            s_out.wait_event(ev["comp"][b])
            with torch.cuda.stream(s_out):
                ulh[b].copy_(uls[b], non_blocking=True)
            ev["out"][b].record(s_out)
        stream.wait_event(ev["out"][(k_steps - 1) % 2])
        stream.wait_event(ev["out"][k_steps % 2])

    e2e_pipelined(4)
    torch.cuda.synchronize()
    barrier()
    p0 = torch.cuda.Event(enable_timing=True)
    p1 = torch.cuda.Event(enable_timing=True)
    s_in.wait_stream(stream)
    p0.record(s_in)
    e2e_pipelined(args.steps)
    p1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(p0.elapsed_time(p1), world, dev)
    e2e_value = world * n / (e2e_ms / args.steps / 1000.0)
    assert torch.equal(ulh[0], ulh[1])               # every step computed the same U
    del xs, fs_, uls

    # ---- step-time distribution (each step bracketed by its own events)
    per_step = []
    for _ in range(args.steps):
        if flush is not None:
            flush.zero_()
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        step()
        a1.record(stream)
        a1.synchronize()
        per_step.append(a0.elapsed_time(a1))
    per_step.sort()
    p50 = per_step[len(per_step) // 2]
    p99 = per_step[min(len(per_step) - 1, int(0.99 * len(per_step)))]

    # ---- the plain FP64 path on the same inputs: throughput and the accuracy
    # of the chosen form against it (the FP64 path matches the oracle: bit for
    # bit in interpolation, to summation order in spread)
    plain = None
    refgpu = None
    if precision != ibk.FP64:
        plan64 = ibk.Plan(ibk.Mac(w.refinement), dom, ibk.Bspline(3), ibk.FP64)
        plan64.reserve(n)
        fe64 = [torch.empty(s_, dtype=torch.float64, device=dev) for s_ in sizes]
        ul64 = torch.empty(3 * n, dtype=torch.float64, device=dev)

        def step64():
            plan64.spread_interpolate(n, x, f, fe64, ue, ul64, stream)

        for _ in range(2):
            step64()
        step()
        barrier()
        err = {"spread_max": 0.0, "spread_rms": 0.0, "interp_max": 0.0, "interp_rms": 0.0}
        # per face: |err| / sum over the face's terms of |res w F| (the FP64
        # spread of |F|: bspline<3> weights are non-negative)
        fa64 = [torch.empty(s_, dtype=torch.float64, device=dev) for s_ in sizes]
        plan64.spread(n, x, f.abs(), fa64, stream)
        face = {}
        for c in range(3):
            touched = fa64[c] > 0
            rel = ((fe[c] - fe64[c]).abs()[touched] / fa64[c][touched]).sort().values
            big = fa64[c] >= 1e-6 * float(fa64[c].max())
            rel_big = ((fe[c] - fe64[c]).abs()[big] / fa64[c][big]).sort().values
            for key, r in (("all", rel), ("significant", rel_big)):
                m = r.numel()
                stats = {q: float(r[min(m - 1, int(q * m))]) for q in (0.5, 0.9, 0.99, 0.999)}
                stats["max"] = float(r[-1])
                prev = face.get(key)
                face[key] = stats if prev is None else {k: max(prev[k], v) for k, v in stats.items()}
            del rel, rel_big, touched, big
        del fa64
        for c in range(3):
            ref_f = fe64[c]
            scale = float(ref_f.abs().max())
            d = (fe[c] - ref_f)
            err["spread_max"] = max(err["spread_max"], float(d.abs().max()) / scale)
            err["spread_rms"] = max(err["spread_rms"], float(d.square().mean().sqrt()) / float(ref_f.square().mean().sqrt()))
            ref_u = ul64[c * n:(c + 1) * n]
            du = ul[c * n:(c + 1) * n] - ref_u
            err["interp_max"] = max(err["interp_max"], float(du.abs().max()) / float(ref_u.abs().max()))
            err["interp_rms"] = max(err["interp_rms"], float(du.square().mean().sqrt()) / float(ref_u.square().mean().sqrt()))
        k64 = max(3, args.steps // 2)
        b0 = torch.cuda.Event(enable_timing=True)
        b1 = torch.cuda.Event(enable_timing=True)
        b0.record(stream)
        for _ in range(k64):
            step64()
        b1.record(stream)
        torch.cuda.synchronize()
        ms64 = b0.elapsed_time(b1) / k64
        plain = {"value": world * n / (ms64 / 1000.0), "unit": "points/s", "ms_per_step": ms64,
                 "steps": k64, "speedup": ms64 / ms_step,
                 "accuracy_vs_fp64": {k: v for k, v in err.items()},
                 "accuracy_note": "normwise: max|err|/max|ref| and rms(err)/rms(ref), worst component",
                 "spread_error_per_face": {
                     "all_touched_faces": face["all"],
                     "faces_with_sum_above_1e-6_of_max": face["significant"],
                     "note": ("|err| / sum over the face's terms of |res w F|, quantiles over faces, worst "
                              "component; a face reached only by far stencil tails sums to less than the "
                              "fixed-point unit of its tile (2^-22 of the tile's largest term) and reads 0")}}
        # the reference's algorithm restated on the GPU, on the same inputs
        if world == 1:
            r = run_reference_gpu(ibk, w, plan64.info, x, f, ue)
            if r is not None:
                dev_s = max(float((a - b).abs().max()) / max(float(b.abs().max()), 1e-300)
                            for a, b in zip(r["fe"], fe64))
                dev_u = float((r["ul"] - ul64).abs().max())
                refgpu = {k: v for k, v in r.items() if k not in ("fe", "ul")}
                refgpu["speedup_of_fp32c"] = r["ms_per_step"] / ms_step
                refgpu["speedup_of_fp64"] = r["ms_per_step"] / ms64
                refgpu["agreement_with_fp64"] = {"spread_max_rel": dev_s, "interp_max_abs": dev_u}
                del r
        del fe64, ul64, plan64

    extras = {}
    if not args.no_extras and args.leg == "all":
        del fe, ul
        torch.cuda.empty_cache()
        extras["batched"] = run_batched(ibk, W, dev, seed=0, steps=max(5, args.steps // 2), rank=rank, world=world)
        extras["serving"] = run_serving(ibk, W, dev, seed=rank, rates=[1000, 2000, 5000, 10000, 20000, 50000])
        extras["membrane"] = run_membrane(ibk, dev, steps=max(5, args.steps // 2))
        extras["fluid"] = run_fluid(ibk, W, dev, steps=3)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_measure(w)
        cpu = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": "points/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32",
        "data": "synthetic (seeded RBC / platelet surfaces, iid N(0,1) forces and velocities)",
        "config": dict(workload_config(w, args.precision), parallelism=f"replicas{world}"),
        "faces_per_s": world * G / (ms_step / 1000.0),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "traffic_source": traffic_source,
                     "kernel": name,
                     "algorithmic_bytes_per_launch": op_bytes, "avg_launch_ms": avg_ms,
                     "peak_source": peak_kind},
        "kernels": kernels,
        "e2e": {"value": e2e_value, "unit": "points/s", "h2d_bytes_per_step": 2 * 8 * 3 * n,
                "d2h_bytes_per_step": 8 * 3 * n,
                "serial_value": e2e_serial,
                "note": ("x and F copied in from pinned host memory and U copied out every step through the "
                         "public API, grid fields device-resident; value: uploads, compute and downloads of "
                         "consecutive steps overlapped on two copy streams; serial_value: one step after the "
                         "other")},
        "p50_ms": p50, "p99_ms": p99,
        "plain_fp64": plain,
        "reference_algorithm_gpu": refgpu,
        "gpu_launches": launches,
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    line.update(extras)
    print(json.dumps(line), flush=True)


# ------------------------------------- the reference's algorithm on the GPU
REFGPU_LIB = os.path.join(ROOT, "baseline", "ref_gpu", "lib", "librefgpu.so")


def grid_geom_struct(info, lengths, boundaries):
    """The library's device GridGeom for a grid, from ibk_grid_info (same
    values and IEEE operations as the library's host geometry)."""
    import ctypes

    class CompGeom(ctypes.Structure):
        _fields_ = [("points", ctypes.c_int * 3), ("cells", ctypes.c_int * 3),
                    ("shift", ctypes.c_double * 3), ("s_over_r", ctypes.c_double * 3),
                    ("size", ctypes.c_longlong)]

    class GridGeom(ctypes.Structure):
        _fields_ = [("dims", ctypes.c_int), ("solid", ctypes.c_int * 3), ("length", ctypes.c_double * 3),
                    ("length_safe", ctypes.c_double * 3), ("r", ctypes.c_double), ("res", ctypes.c_double),
                    ("comp", CompGeom * 3)]

    g = GridGeom()
    dims = info.dims
    g.dims = dims
    r = info.resolution
    g.r = r
    res = 1.0
    for _ in range(dims):
        res = r * res
    g.res = res
    for d in range(dims):
        g.solid[d] = 0 if boundaries[d] == 0 else 1
        g.length[d] = lengths[d]
        g.length_safe[d] = lengths[d] * (1.0 - 2.0 ** -52)
    for c in range(dims):
        cg = g.comp[c]
        for d in range(dims):
            cg.points[d] = info.points[c][d]
            cg.cells[d] = info.cells[c][d]
            cg.shift[d] = info.shift[c][d]
            cg.s_over_r[d] = info.shift[c][d] / r
        cg.size = info.size[c]
    return g


def run_reference_gpu(ibk, w, info, x, f, ue, steps=5):
    """Times the GPU restatement of the reference's own algorithm (sort by
    cell key, 8 sweeps of segmented sums into 8 planes, plane combine;
    per-point gathers for interpolation) on the same inputs, FP64, on the
    legacy default stream as the reference runs.  None when its library is
    not built."""
    import ctypes
    import torch
    if not os.path.exists(REFGPU_LIB):
        return None
    L = ctypes.CDLL(REFGPU_LIB)
    L.refgpu_spread.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                ctypes.POINTER(ctypes.c_void_p)]
    L.refgpu_interpolate.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                     ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p]
    L.refgpu_last_error.restype = ctypes.c_char_p
    g = grid_geom_struct(info, w.lengths, w.boundaries)
    n = w.n
    dev = x.device
    fe = [torch.empty(int(info.size[c]), dtype=torch.float64, device=dev) for c in range(3)]
    ul = torch.empty(3 * n, dtype=torch.float64, device=dev)
    fp = (ctypes.c_void_p * 3)(*[a.data_ptr() for a in fe])
    up = (ctypes.c_void_p * 3)(*[a.data_ptr() for a in ue])
    default = torch.cuda.default_stream(dev)

    def step():
        if L.refgpu_spread(ctypes.byref(g), n, x.data_ptr(), f.data_ptr(), fp) != 0:
            raise RuntimeError(L.refgpu_last_error().decode())
        if L.refgpu_interpolate(ctypes.byref(g), n, x.data_ptr(), up, ul.data_ptr()) != 0:
            raise RuntimeError(L.refgpu_last_error().decode())

    torch.cuda.synchronize()
    step()
    torch.cuda.synchronize()
    times = []
    for _ in range(steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(default)
        step()
        e1.record(default)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    ms = statistics.median(times)
    return {"value": n / (ms / 1000.0), "unit": "points/s", "ms_per_step": ms, "steps": steps,
            "ms_min": min(times), "ms_max": max(times),
            "fe": fe, "ul": ul,
            "note": ("GPU restatement of the reference's algorithm, labelled as such (its own CUDA build does "
                     "not compile with nvcc 12.9): per component a sort of the points by cell key (Thrust), "
                     "a unique count with a host sync, 8 sweeps of weights, segmented sums (Thrust "
                     "reduce_by_key) and plane scatters, a combine over 8 planes; interpolation as one thread "
                     "per point gathering 64 nodes; FP64, temporaries allocated per call as the reference does "
                     "(their cudaMalloc / cudaFree are inside the timed steps); median step")}


# ------------------------------------------------ batched and serving legs
def ensemble_arrays(ibk, W, insts_w, precision, dev, seed):
    """Batch + device arrays of an ensemble (one dict per instance)."""
    import torch
    insts = [ibk.Instance(ibk.Mac(w.refinement),
                          ibk.Domain(*[ibk.Dimension(l, b) for l, b in zip(w.lengths, w.boundaries)]))
             for w in insts_w]
    total = sum(w.n for w in insts_w)
    batch = ibk.Batch(insts, ibk.Bspline(3), precision, max_points=total)
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    io = []
    for i, w in enumerate(insts_w):
        sizes = batch.sizes(i)
        io.append({"n": w.n, "x": torch.from_numpy(w.x).to(dev), "fl": torch.from_numpy(w.f).to(dev),
                   "ue": [torch.randn(s_, generator=gen, dtype=torch.float64, device=dev) * W.UM_PER_S
                          for s_ in sizes],
                   "fe": [torch.empty(s_, dtype=torch.float64, device=dev) for s_ in sizes],
                   "ul": torch.empty(3 * w.n, dtype=torch.float64, device=dev)})
    batch.bind(io)
    return batch, io, total


def time_batch(batch, ops, steps, stream):
    import torch
    for _ in range(3):
        for op in ops:
            batch.run(op, stream)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        for op in ops:
            batch.run(op, stream)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def run_batched(ibk, W, dev, seed, steps, rank=0, world=1):
    """256 independent instances (cube grids of 32^3..128^3, 1-50 cells), one
    persistent graph-captured launch per operator; FP32C vs FP64 batches and
    a loop of single plans for comparison.  With several ranks the 256
    instances are partitioned over them (longest first; no exchange), each
    rank runs its share, and the times are the slowest rank's."""
    import torch
    from ib_cu_b200 import sharding
    stream = torch.cuda.current_stream()
    everything = W.ensemble(seed=seed, count=256)
    # periodic cubes of side s cells: 3 s^3 faces (h = 0.25 um = 0.025 units)
    cube_faces = [3 * int(round(w.lengths[0] / 0.025)) ** 3 for w in everything]
    shards = sharding.partition([sharding.instance_cost(w.n, f) for w, f in zip(everything, cube_faces)], world)
    insts_w = [everything[i] for i in shards[rank]]
    ops = (ibk.OP_SPREAD_INTERPOLATE,)      # spread and interpolation, one binning
    out = {"instances": len(everything), "instances_this_rank": len(insts_w),
           "scaling": "strong", "parallelism": f"instances partitioned over {world} rank(s)"}
    batch, io, total = ensemble_arrays(ibk, W, insts_w, ibk.FP32C, dev, 2000 + seed)
    faces = sum(cube_faces)
    assert world > 1 or faces == sum(sum(batch.sizes(i)) for i in range(len(insts_w)))
    t_default = max_over_ranks(time_batch(batch, ops, steps, stream), world, dev)
    cfg = batch.tune(ibk.OP_SPREAD_INTERPOLATE, stream)
    for op in ops:
        batch.capture(op)
    l0 = batch.launch_count()
    ms = max_over_ranks(time_batch(batch, ops, steps, stream), world, dev)
    launches = (batch.launch_count() - l0) // (steps + 3)
    all_points = sum(w.n for w in everything)
    out.update({"points": all_points, "faces": faces, "value": all_points / (ms / 1000.0), "unit": "points/s",
                "ms_per_step": ms, "faces_per_s": faces / (ms / 1000.0), "ms_default_config": t_default,
                "tuned_config": cfg, "launches_per_step": launches,
                "roofline_bytes_per_step": 2 * algorithmic_bytes(total, faces)})
    # FP64 batch (the plain path, batched) on the same inputs
    b64 = ibk.Batch([ibk.Instance(ibk.Mac(w.refinement),
                                  ibk.Domain(*[ibk.Dimension(l, b_) for l, b_ in zip(w.lengths, w.boundaries)]))
                     for w in insts_w], ibk.Bspline(3), ibk.FP64, max_points=total)
    fe64 = [[torch.empty_like(a) for a in e["fe"]] for e in io]
    ul64 = [torch.empty_like(e["ul"]) for e in io]
    b64.bind([dict(e, fe=fe64[i], ul=ul64[i]) for i, e in enumerate(io)])
    for op in ops:
        b64.capture(op)
    ms64 = max_over_ranks(time_batch(b64, ops, max(3, steps // 2), stream), world, dev)
    err_s = err_u = 0.0
    for i, e in enumerate(io):
        for c in range(3):
            ref = fe64[i][c]
            err_s = max(err_s, float((e["fe"][c] - ref).abs().max()) / max(float(ref.abs().max()), 1e-300))
        n_i = e["n"]
        for c in range(3):
            ref = ul64[i][c * n_i:(c + 1) * n_i]
            err_u = max(err_u, float((e["ul"][c * n_i:(c + 1) * n_i] - ref).abs().max())
                        / max(float(ref.abs().max()), 1e-300))
    out["plain_fp64"] = {"value": all_points / (ms64 / 1000.0), "ms_per_step": ms64, "speedup": ms64 / ms,
                         "accuracy_vs_fp64": {"spread_max": err_s, "interp_max": err_u}}
    del b64, fe64, ul64
    # a loop of single FP32C plans (one per instance), for the batching gain
    plans = [ibk.Plan(ibk.Mac(w.refinement),
                      ibk.Domain(*[ibk.Dimension(l, b_) for l, b_ in zip(w.lengths, w.boundaries)]),
                      ibk.Bspline(3), ibk.FP32C) for w in insts_w]

    def loop():
        for p_, e in zip(plans, io):
            p_.spread_interpolate(e["n"], e["x"], e["fl"], e["fe"], e["ue"], e["ul"], stream)

    for _ in range(2):
        loop()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(max(2, steps // 4)):
        loop()
    e1.record(stream)
    torch.cuda.synchronize()
    ms_loop = max_over_ranks(e0.elapsed_time(e1) / max(2, steps // 4), world, dev)
    out["plan_loop"] = {"ms_per_step": ms_loop, "batch_speedup": ms_loop / ms}
    del plans, batch, io
    torch.cuda.empty_cache()
    return out


def run_membrane(ibk, dev, steps, nc=64, ns=10000, nd=2500, warmup=3):
    """Membrane forces of nc shapes with the reference's RBC discretisation
    (rbc{2500, 10000}: 2500 data sites, 10000 sample sites,
    test/ib-whole.cc:233): per step the current geometry (six FP64 operator
    products of ns x nd operators with the 3*nc position columns, then the
    per-sample normal and patch area) and the Skalak tension from it and the
    rest geometry (computed once), then the bending force (the curvature field
    at the data sites through the data-site operators, its derivatives at the
    samples), then the viscous dissipation (the velocity's five derivatives
    at the samples, then the per-sample stress divergence): the reference's
    red-cell force set (test/ib-whole.cc:210-213).  Random operators,
    positions and velocities of the reference's shapes: the timing does not
    depend on their values."""
    import torch
    gen = torch.Generator(device=dev)
    gen.manual_seed(11)
    ops = [torch.randn(ns, nd, generator=gen, dtype=torch.float64, device=dev) / nd for _ in range(6)]
    wts = torch.rand(ns, generator=gen, dtype=torch.float64, device=dev) + 0.5
    plan = ibk.SurfacePlan(ops, wts)
    dops = [None] + [torch.randn(nd, nd, generator=gen, dtype=torch.float64, device=dev) / nd for _ in range(5)]
    dplan = ibk.SurfacePlan(dops, torch.rand(nd, generator=gen, dtype=torch.float64, device=dev) + 0.5)
    del ops, dops
    x0 = torch.randn(3 * nd * nc, generator=gen, dtype=torch.float64, device=dev)
    x1 = x0 + 0.01 * torch.randn(3 * nd * nc, generator=gen, dtype=torch.float64, device=dev)
    rest = plan.geometry(x0, nc)
    vel = torch.randn(3 * nd * nc, generator=gen, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
    geo_ms, ten_ms, ben_ms, dis_ms = [], [], [], []
    for it in range(warmup + steps):
        ev[0].record(stream)
        cur = plan.geometry(x1, nc)
        ev[1].record(stream)
        f = ibk.membrane_tension(ibk.SKALAK, 0.25, 25.0, rest, cur)
        ev[2].record(stream)
        fb = ibk.membrane_bending(dplan, plan, 1.0, False, None, x1, None, cur, nc)
        ev[3].record(stream)
        fd = ibk.membrane_dissipation(plan, 0.25, vel, cur, nc)
        ev[4].record(stream)
        torch.cuda.synchronize()
        if it >= warmup:
            geo_ms.append(ev[0].elapsed_time(ev[1]))
            ten_ms.append(ev[1].elapsed_time(ev[2]))
            ben_ms.append(ev[2].elapsed_time(ev[3]))
            dis_ms.append(ev[3].elapsed_time(ev[4]))
        del cur, f, fb, fd
    g, t, b = float(np.median(geo_ms)), float(np.median(ten_ms)), float(np.median(ben_ms))
    d = float(np.median(dis_ms))
    bflops = (5 * 2.0 * nd * nd * 3 * nc) + (5 * 2.0 * ns * nd * nc)
    dflops = 5 * 2.0 * ns * nd * 3 * nc
    flops = 6 * 2.0 * ns * nd * 3 * nc
    tbytes = (2 * 15 + 1 + 3) * 8.0 * ns * nc     # rest t, tt and area + current t, tt read; f written
    peak, _ = measured_peaks()
    del plan, dplan, rest, vel
    torch.cuda.empty_cache()
    return {"shapes": nc, "data_sites": nd, "samples": ns, "law": "skalak", "steps": steps,
            "ms_per_step": g + t + b + d, "geometry_ms": g, "tension_ms": t, "bending_ms": b,
            "dissipation_ms": d, "dissipation_tflops": dflops / (d * 1e-3) / 1e12,
            "bending_gemm_tflops": bflops / (b * 1e-3) / 1e12,
            "geometry_tflops": flops / (g * 1e-3) / 1e12,
            "tension_gbs": tbytes / (t * 1e-3) / 1e9, "tension_frac_of_hbm": tbytes / (t * 1e-3) / 1e9 / peak,
            "note": "FP64: operator products as library DGEMMs, normal / area and tension as hand-written "
                    "kernels; median of the timed steps, CUDA events"}


def run_fluid(ibk, W, dev, steps, warmup=1, workload="large-channel"):
    """The fluid step that consumes the spread's force density: one implicit
    diffusion step (Crank-Nicolson, gamma = 1) of the x-velocity grid of the
    large channel (512 x 256 x 512 cells, walls in y: Dirichlet; or another
    channel workload's grid), mu = 1, timestep 1e-3 (internal units: mu k /
    h^2 = 1.6), solver tolerance 1e-11 as the reference's drivers set it.
    Random velocity, force and rhs."""
    import torch
    w = make_workload(workload)
    dom = ibk.Domain(*[ibk.Dimension(l, b) for l, b in zip(w.lengths, w.boundaries)])
    plan = ibk.Plan(ibk.Mac(w.refinement), dom, ibk.Bspline(3), ibk.FP64)
    d = ibk.Diffusion(plan, 0, 1e-3, 1.0, tolerance=1e-11, max_iterations=5000)
    gen = torch.Generator(device=dev)
    gen.manual_seed(17)
    u, f, rhs = (torch.randn(d.size, generator=gen, dtype=torch.float64, device=dev) for _ in range(3))
    times, its = [], []
    for it in range(warmup + steps):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        out = d.step(u, rhs, f, gamma=1.0)
        e1.record()
        torch.cuda.synchronize()
        if it >= warmup:
            times.append(e0.elapsed_time(e1))
            its.append(d.iterations)
        del out
    ms = float(np.median(times))
    iters = int(np.median(its))
    # Chebyshev-preconditioned iteration, bytes per face: operator (d in, q
    # out: 16), x / r update (48), the three polynomial steps (16 + 24 + 24),
    # direction (24)
    per_iter_bytes = 152.0 * d.size
    peak, _ = measured_peaks()
    res = {"faces": d.size, "grid": "x".join(str(int(round(l / 0.025))) for l in w.lengths) + " (x faces)",
           "steps": steps, "ms_per_step": ms,
           "iterations": iters, "ms_per_iteration": ms / max(iters, 1),
           "iteration_gbs": per_iter_bytes * iters / (ms * 1e-3) / 1e9,
           "iteration_frac_of_hbm": per_iter_bytes * iters / (ms * 1e-3) / 1e9 / peak,
           "note": "FP64 matrix-free operator and PCG with the reference's degree-4 Chebyshev preconditioner "
                   "(Gershgorin interval), the convergence test read back once per iteration; median of the "
                   "timed steps, CUDA events"}
    del d, plan, u, f, rhs
    torch.cuda.empty_cache()
    return res


def run_serving(ibk, W, dev, seed, rates, seconds_per_rate=1.0, slots=4, slot_sweep=(1, 2, 8), sweep_rate=50000):
    """Serving sweep: 256 ensemble members resident on the device, Poisson
    step requests (interpolate, advect dt = 1 us, spring k = 1 pN/um,
    spread) at each offered rate, continuous batching on `slots` streams;
    then the saturating rate again with other slot counts.  Each launch's
    host time (packing the ready members, binding, launching) is reported."""
    insts_w = W.ensemble(seed=seed, count=256)
    doms = [ibk.Domain(*[ibk.Dimension(l, b) for l, b in zip(w.lengths, w.boundaries)]) for w in insts_w]
    insts = [ibk.Instance(ibk.Mac(w.refinement), d) for w, d in zip(insts_w, doms)]
    dt = 1e-6 * 1e3            # 1 us in the internal time unit (1 ms)
    k = W.PN / W.UM            # 1 pN/um
    rng = np.random.default_rng(3000 + seed)
    velocities = [[rng.normal(size=s_) * W.UM_PER_S
                   for s_ in ibk.Plan(ibk.Mac(w.refinement), d, ibk.Bspline(3), ibk.FP32C).sizes()]
                  for w, d in zip(insts_w, doms)]

    def server(nslots):
        srv = ibk.Server(insts, ibk.Bspline(3), ibk.FP32C, slots=nslots, dt=dt, k=k,
                         hbm_budget=150 * 10**9, max_points=sum(w.n for w in insts_w))
        for i, w in enumerate(insts_w):
            srv.admit(i, w.x, velocities[i])
        srv.run_poisson(rate=500.0, requests=100, seed=1)          # warm-up
        return srv

    def entry(r, st):
        return {"offered_per_s": r, "requests": st["requests"], "p50_ms": st["p50_ms"],
                "p99_ms": st["p99_ms"], "mean_ms": st["mean_ms"],
                "served_per_s": st["requests"] / max(st["wall_s"], 1e-9),
                "points_per_s": st["points"] / max(st["wall_s"], 1e-9),
                "launches": st["launches"], "host_ms_per_launch": st["host_ms_per_launch"]}

    srv = server(slots)
    sweep = []
    for r in rates:
        nreq = int(max(200, min(20000, r * seconds_per_rate)))
        sweep.append(entry(r, srv.run_poisson(rate=float(r), requests=nreq, seed=int(r))))
    admitted = srv.stats()["admitted_bytes"]
    srv.close()
    slots_sweep = []
    for ns_ in slot_sweep:
        srv = server(ns_)
        e = entry(sweep_rate, srv.run_poisson(rate=float(sweep_rate), requests=10000, seed=7))
        e["slots"] = ns_
        slots_sweep.append(e)
        srv.close()
    return {"members": len(insts_w), "slots": slots, "admitted_bytes": admitted,
            "hbm_budget_bytes": 150 * 10**9, "sweep": sweep, "slot_sweep": slots_sweep}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="large-channel",
                    choices=["large-channel", "medium-channel", "channel", "single-rbc"])
    ap.add_argument("--precision", choices=["fp32c", "fp64"], default="fp32c")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--leg", choices=["all", "batched", "serving", "membrane", "fluid"], default="all",
                    help="batched / serving / membrane / fluid: run that leg alone (its own JSON line)")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batched (256 instances) and serving legs")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
