"""Benchmark of the splat depth-key + stable counting sort on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--workload mixed-64|clusters-1M|uniform-100k|slab-6M] [--cull C]

One step is one pass of the sort over one batch of synthetic splats. The
default workload, mixed-64, is 64 (scene, view) jobs of 10k-2M splats (25M in
all, cull 0.5), every job's cloud resident in HBM; one step is one
graph-captured launch of the batch (ws_plan_launch: the counters reset, the
keys kernel and the two digit passes over all 64 jobs; the job table with the
views stays resident, uploaded by ws_plan_set_views).
Prints one JSON line:

  value        Msplats/s (whole job, all ranks), outputs to device memory,
               CUDA events on the launching stream, L2 flushed (a 256 MiB
               write) before every timed step
  e2e          the same metric through the public batch call with host
               outputs (ws_sort_batch_host): per step every job's survivor
               count and order come back to pinned host memory; the bytes
               each way are the library's own copy counters
  roofline     32 N + 8 S summed over the jobs / the sort kernels' event-timed
               duration, against the measured HBM copy bandwidth
  cpu_baseline the CPU oracle (C++ restatement of the reference's path, all
               host threads) on a bounded sample of the same jobs
  batch        the same 64 jobs as 64 plain ws_sort calls, as one ws_sort_batch
               call and as the graph launch
  suite        the other measured targets: clusters-1M and slab-6M as plain
               single-cloud sorts, the served stream, particles, shading,
               decoding and drawing

--workload clusters-1M (or uniform-100k, slab-6M) makes one plain ws_sort of
that cloud the step instead. --impl reference times the reference's
algorithm on the host CPU over the same jobs (the oracle port; the
reference's own JavaScript needs Node, which this machine does not have) and
prints the same line with "impl": "reference". With N > 1 (torchrun) every
rank sorts its own batch of 64 jobs (other seeds), weak scaling with no
collective on the data path; the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FALLBACK_HBM_GBS = 6650.0
ALGORITHMS = ("three-phase", "one-CTA radix", "one-CTA counting")
L2_FLUSH_BYTES = 256 << 20


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="wsort", choices=["wsort", "reference"])
    ap.add_argument("--workload", default="mixed-64",
                    choices=["mixed-64", "clusters-1M", "uniform-100k", "slab-6M"])
    ap.add_argument("--cull", type=float, default=0.5)
    ap.add_argument("--no-suite", action="store_true", help="skip the side measurements")
    ap.add_argument("--cpu-seconds", type=float, default=10.0, help="CPU baseline sample length")
    ap.add_argument("--tile", type=int, default=0,
                    help="fixed least splats a segment covers (skips the autotuner; with --ctas)")
    ap.add_argument("--ctas", type=int, default=0, help="fixed kernel variant: 1 or 2 CTAs per SM (with --tile)")
    ap.add_argument("--segs", type=int, default=1, help="fixed segments per resident CTA (with --tile)")
    ap.add_argument("--only", default="", choices=["", "particles-64", "shade-1M", "decode", "draw-1M", "sort-batch"],
                    help="run one side measurement alone and print its result (no bench line); sort-batch: "
                         "mixed-64 as 3 + 3 batched launches with the --tile/--ctas/--segs parameters (for a "
                         "profiler: the 4th launch's three kernels are launches 9-11)")
    return ap.parse_args()


def peak_hbm():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic(workload: str, cull: float):
    """DRAM bytes per launch of the sort kernel from the committed ncu summary
    (profiles/sort_kernel_traffic.txt: `<workload> <cull> <bytes>` lines), or None."""
    path = os.path.join(ROOT, "profiles", "sort_kernel_traffic.txt")
    try:
        for line in open(path):
            parts = line.split()
            if len(parts) >= 3 and not line.startswith("#") and parts[0] == workload and float(parts[1]) == cull:
                return int(float(parts[2]))
    except OSError:
        pass
    return None


def make_jobs(workload: str, cull: float, seed_offset: int = 0):
    from winding_b200 import workloads as W
    if workload == "clusters-1M":
        return [W.clusters_1m(seed=1 + seed_offset, cull=cull)]
    if workload == "uniform-100k":
        return [W.uniform_100k(seed=0 + seed_offset, cull=cull)]
    if workload == "slab-6M":
        return [W.slab_6m(seed=2 + seed_offset, cull=cull)]
    return W.mixed_64(seed=3 + seed_offset, cull=cull)


class Clocks:
    """nvidia-smi samples of the SM clock and throttle reasons during a region."""

    FIELDS = "clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown," \
             "clocks_event_reasons.sw_power_cap"

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax = float(parts[1])
            except ValueError:
                continue
            for name, flag in zip(names, parts[4:8]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_baseline(jobs, seconds: float, threads: int, runs: int = 5):
    """The oracle on the host cores: after a warm-up sort, `runs` timed runs of
    about seconds / runs each, every run sorting full views of the workload in
    turn (continuing where the previous run stopped). Returns (median
    Msplats/s, sample text with the runs' spread)."""
    from oracle import oracle as O
    parsed = [O.parse_splat(j.bytes()) for j in jobs]
    order = sorted(range(len(jobs)), key=lambda k: parsed[k].count)

    def sort(k):
        j = jobs[k]
        O.sort_view(parsed[k], j.view.model_view, j.view.projection, j.view.viewport, j.view.cull, threads=threads)
        return parsed[k].count

    sort(order[0])   # warm-up: the smallest view
    rates, sorts, done_all, at = [], 0, 0, 0
    for _ in range(runs):
        done = 0
        t0 = time.perf_counter()
        while True:
            done += sort(at % len(jobs))
            at += 1
            sorts += 1
            if time.perf_counter() - t0 >= seconds / runs:
                break
        rates.append(done / (time.perf_counter() - t0) / 1e6)
        done_all += done
    med = sorted(rates)[len(rates) // 2]
    return med, (f"median of {runs} runs of ~{seconds / runs:.1f} s ({sorts} full-view sorts, {done_all} splats "
                 f"in all; runs {min(rates):.1f}-{max(rates):.1f} Msplats/s)")


def run_reference(args, rank: int):
    if rank != 0:
        return
    jobs = make_jobs(args.workload, args.cull)
    threads = os.cpu_count() or 1
    # Each step: one full pass of the workload's views on the host cores.
    from oracle import oracle as O
    parsed = [O.parse_splat(j.bytes()) for j in jobs]

    def step():
        n = 0
        for p, j in zip(parsed, jobs):
            O.sort_view(p, j.view.model_view, j.view.projection, j.view.viewport, j.view.cull, threads=threads)
            n += p.count
        return n

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    total = 0
    for _ in range(args.steps):
        total += step()
    dt = time.perf_counter() - t0
    value = total / dt / 1e6
    line = {
        "impl": "reference", "metric": "Msplats/s sorted (bit-exact stable order)", "value": value,
        "unit": "Msplats/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 keys, u32 sort", "data": "synthetic (seeded)",
        "config": {"workload": args.workload, "jobs": len(jobs), "splats_per_step": total // args.steps,
                   "cull": args.cull, "viewport": [1920, 1080]},
        "cpu_baseline": {"value": value, "unit": "Msplats/s", "cores": threads, "kind": "port",
                         "sample": f"{args.steps} steps of the full workload; C++ restatement of the reference's "
                                   f"makeKeys + stable counting sort (the reference's JavaScript needs Node, absent)"},
        "e2e": {"value": value, "unit": "Msplats/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def timed_sorts(ctx, torch, steps, flush, fn, host_start=False):
    """Runs fn() `steps` times, each bracketed by CUDA events on torch's
    current stream with an L2 flush before it. Returns total ms. host_start:
    the flush finishes before the start event is recorded, so a call's host
    work before its first launch is inside the bracket (the end-to-end
    measurements)."""
    stream = torch.cuda.current_stream()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for a, b in evs:
        flush.zero_()
        if host_start:
            stream.synchronize()
        a.record(stream)
        fn()
        b.record(stream)
    torch.cuda.synchronize()
    return sum(a.elapsed_time(b) for a, b in evs)


def load_jobs(ctx, torch, jobs):
    """Each job's cloud resident on the device, its view, and device outputs
    (order, keys, count)."""
    from winding_b200 import make_view, parse_splats
    clouds, outs, views = [], [], []
    for j in jobs:
        sp = parse_splats(j.records, ctx)
        n = max(sp.count, 1)
        o = torch.empty(n, dtype=torch.int32, device="cuda")
        k = torch.empty(n, dtype=torch.int32, device="cuda")
        c = torch.zeros(1, dtype=torch.int32, device="cuda")
        clouds.append(sp)
        outs.append((o, k, c))
        views.append(make_view(j.view.model_view, j.view.projection, j.view.viewport, j.view.cull))
    return {"clouds": clouds, "views": views, "outs": outs, "splats": sum(sp.count for sp in clouds)}


def time_plain(ctx, torch, p, steps, warmup, flush):
    """One plain ws_sort per job (device outputs) per step; fills p's ms,
    kernel_ms, launches and survivors."""
    stream = torch.cuda.current_stream().cuda_stream

    def one():
        for sp, v, (o, k, c) in zip(p["clouds"], p["views"], p["outs"]):
            ctx.sort_device(sp, v, o.data_ptr(), k.data_ptr(), c.data_ptr(), stream)

    for _ in range(warmup):
        one()
    torch.cuda.synchronize()
    ctx.timing(True)
    p["ms"] = timed_sorts(ctx, torch, steps, flush, one)
    p["kernel_ms"], p["launches"] = ctx.timing_read()
    ctx.timing(False)
    p["survivors"] = [int(c.item()) for _, _, c in p["outs"]]
    return p


def plain_measure(ctx, torch, jobs, steps, warmup, flush):
    """Plain ws_sort per job (device outputs). Returns dict with totals."""
    return time_plain(ctx, torch, load_jobs(ctx, torch, jobs), steps, warmup, flush)


def tune_batch(ctx, p, args):
    """The launch parameters: fixed from the command line, or the autotuner's
    choice per size bucket (each bucket's first job alone, and the whole
    batch)."""
    from winding_b200 import autotune
    if args.tile and args.ctas:
        ctx.set_params(tile=args.tile, ctas_per_sm=args.ctas, segs_per_cta=args.segs, algorithm=0)
        return {autotune.bucket(p["splats"]): (args.tile, args.ctas, args.segs, 0)}
    pairs = list(zip(p["clouds"], p["views"]))
    per_bucket = {}
    for pair in pairs:
        per_bucket.setdefault(autotune.bucket(pair[0].count), pair)
    sets = [[pr] for pr in per_bucket.values()]
    if len(pairs) > 1:
        sets.append(pairs)
    return autotune.tune(ctx, sets)


def survivors_at_cull0(ctx, torch, plain):
    """Splats that pass the frustum and faintness tests (the ones whose
    covariance the footprint cull reads): the survivor count at cull 0."""
    from winding_b200 import make_view
    stream = torch.cuda.current_stream().cuda_stream
    out = []
    for sp, v, (o, k, c) in zip(plain["clouds"], plain["views"], plain["outs"]):
        v0 = make_view(np.ctypeslib.as_array(v.model_view), np.ctypeslib.as_array(v.projection),
                       (v.viewport[0], v.viewport[1]), 0.0)
        ctx.sort_device(sp, v0, o.data_ptr(), k.data_ptr(), c.data_ptr(), stream)
        torch.cuda.synchronize()
        out.append(int(c.item()))
    return out


def algorithmic_bytes(n, s):
    """The per-(cloud, view) figure the roofline uses: every 32-byte .splat
    record read once and a u32 index plus a u32 key written per survivor,
    32 N + 8 S."""
    return 32 * n + 8 * s


def layout_bytes(n, n_front, s, cull):
    """The same work in the resident layout the reference's GPU path (and
    this library) keeps: each splat's 16-byte centre, the 24-byte covariance
    of every splat the footprint cull examines (cull > 0), and 8 bytes per
    survivor."""
    return 16 * n + (24 * n_front if cull > 0 else 0) + 8 * s


def run_wsort(args, rank, world, local_rank):
    import torch
    torch.cuda.set_device(local_rank)
    # One explicit stream for the flush, the sorts and the events.
    with torch.cuda.stream(torch.cuda.Stream()):
        _run_wsort(args, rank, world, local_rank, torch)


def _run_wsort(args, rank, world, local_rank, torch):
    from winding_b200 import Context
    dist = None
    if world > 1:
        import torch.distributed as dist
    ctx = Context(local_rank)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device="cuda")
    if args.only:   # one side measurement alone (for a profiler, say)
        fns = {"particles-64": particles_suite, "shade-1M": shade_suite, "decode": decode_suite,
               "draw-1M": draw_suite, "sort-batch": lambda c, t, f, pk: sort_batch_only(c, t, f, args)}
        peak, _ = peak_hbm()
        result = fns[args.only](ctx, torch, flush, peak)
        if rank == 0:
            print(json.dumps({"only": args.only, "result": result}), flush=True)
        return
    if args.workload == "mixed-64":
        line, jobs = batch_line(args, rank, world, dist, ctx, torch, flush)
    else:
        line, jobs = single_line(args, rank, world, dist, ctx, torch, flush)
    if rank == 0:
        if world == 1:
            v, sample = cpu_baseline(jobs, args.cpu_seconds, os.cpu_count() or 1)
            v1, sample1 = cpu_baseline(jobs, max(args.cpu_seconds / 3, 1.0), 1)
            line["cpu_baseline"] = {"value": v, "unit": "Msplats/s", "cores": os.cpu_count() or 1, "kind": "port",
                                    "sample": sample + "; C++ restatement of the reference's makeKeys + stable "
                                                       "counting sort, all host threads",
                                    "single_thread": {"value": v1, "unit": "Msplats/s", "cores": 1,
                                                      "sample": sample1 + ", one thread (the reference's "
                                                                          "JavaScript runs on one)"}}
        if not args.no_suite and world == 1:
            try:
                line["suite"] = suite(ctx, torch, flush, args)
            except Exception as exc:   # the headline line still prints
                line["suite"] = {"error": f"{type(exc).__name__}: {exc}"}
        print(json.dumps(line), flush=True)
    ctx.close()


def sort_batch_only(ctx, torch, flush, args):
    """mixed-64 as batched launches (ws_sort_batch) with fixed parameters:
    3 untimed, then 3 timed by the library's kernel events."""
    p = load_jobs(ctx, torch, make_jobs("mixed-64", args.cull))
    ctx.set_params(tile=args.tile or 2048, ctas_per_sm=args.ctas or 1, segs_per_cta=args.segs, algorithm=0)
    stream = torch.cuda.current_stream().cuda_stream
    specs = [(sp, v, o.data_ptr(), k.data_ptr(), c.data_ptr())
             for sp, v, (o, k, c) in zip(p["clouds"], p["views"], p["outs"])]
    for _ in range(3):
        flush.zero_()
        ctx.sort_batch(specs, stream)
    ctx.timing(True)
    timed_sorts(ctx, torch, 3, flush, lambda: ctx.sort_batch(specs, stream))
    kms, launches = ctx.timing_read()
    ctx.timing(False)
    ctx.sync()
    out = {"jobs": len(specs), "splats": p["splats"], "kernel_us": kms / max(launches, 1) * 1e3,
           "params": [args.tile or 2048, args.ctas or 1, args.segs]}
    for sp in p["clouds"]:
        sp.destroy()
    return out


def max_over_ranks(dist, torch, ms):
    t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def batch_line(args, rank, world, dist, ctx, torch, flush):
    """The default step: the 64 mixed jobs as one graph-captured launch."""
    jobs = make_jobs("mixed-64", args.cull, seed_offset=rank)   # each rank its own batch: weak scaling
    p = load_jobs(ctx, torch, jobs)
    time_plain(ctx, torch, p, 0, 1, flush)   # warm
    tuned = tune_batch(ctx, p, args)
    stream = torch.cuda.current_stream().cuda_stream
    specs = [(sp, v, o.data_ptr(), k.data_ptr(), c.data_ptr())
             for sp, v, (o, k, c) in zip(p["clouds"], p["views"], p["outs"])]
    plan = ctx.plan(specs)
    for _ in range(args.warmup):
        plan.launch(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local_rank_of(torch))
    clocks.start()
    ms = timed_sorts(ctx, torch, args.steps, flush, lambda: plan.launch(stream))
    clk = clocks.stop()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ms_max = max_over_ranks(dist, torch, ms)
    plan.close()
    total = p["splats"]
    survivors = [int(c.item()) for _, _, c in p["outs"]]
    value = total * world * args.steps / (ms_max / 1e3) / 1e6

    # The same launch through ws_sort_batch, its three kernels bracketed by
    # the library's timing events: the kernel time of the roofline.
    reps = 10
    for _ in range(2):
        ctx.sort_batch(specs, stream)
    ctx.timing(True)
    b_ms = timed_sorts(ctx, torch, reps, flush, lambda: ctx.sort_batch(specs, stream))
    kms, launches = ctx.timing_read()
    ctx.timing(False)
    kernel_s = kms / max(launches, 1) / 1e3

    # End to end through the public batch call: every job's count and order
    # into pinned host memory, every step.
    host = [(torch.empty(max(sp.count, 1), dtype=torch.int32).pin_memory(), torch.zeros(1, dtype=torch.int32)
             .pin_memory()) for sp in p["clouds"]]
    hspecs = [(sp, v, ho.data_ptr(), None, hc.data_ptr()) for sp, v, (ho, hc) in zip(p["clouds"], p["views"], host)]
    for _ in range(2):
        ctx.sort_batch_host(hspecs, stream)
    e2e_steps = max(3, min(args.steps, 20))
    ctx.copy_stats(reset=True)
    e2e_ms = timed_sorts(ctx, torch, e2e_steps, flush, lambda: ctx.sort_batch_host(hspecs, stream), host_start=True)
    h2d, d2h = ctx.copy_stats(reset=True)
    e2e_ms = max_over_ranks(dist, torch, e2e_ms)
    e2e_single = total * world * e2e_steps / (e2e_ms / 1e3) / 1e6
    assert all(int(hc[0]) == s for (_, hc), s in zip(host, survivors))
    # Pipelined: the same call from two host threads, each with its own
    # context (its own resident copy of the clouds) and stream, steps
    # alternating, so one step's copy to the host overlaps the next step's
    # sort. Every step still brings back every job's count and order.
    pipe_steps = 2 * max(3, min(args.steps, 20) // 2)
    pipe_ms, pipe_h2d, pipe_d2h = pipelined_e2e(ctx, torch, jobs, p, tuned, pipe_steps)
    pipe_ms = max_over_ranks(dist, torch, pipe_ms)
    e2e_value = total * world * pipe_steps / (pipe_ms / 1e3) / 1e6

    line = {
        "metric": "Msplats/s sorted (bit-exact stable order)", "value": value, "unit": "Msplats/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 keys, u32 sort", "data": "synthetic (seeded)",
        "config": {"workload": "mixed-64", "jobs": len(jobs), "splats_per_step": total * world,
                   "survivors_per_step": sum(survivors), "job_splats": [10_000, 2_000_000], "cull": args.cull,
                   "viewport": [1920, 1080], "l2": "flushed (256 MiB write) before each step",
                   "launch": "ws_plan_launch: one graph (counter reset, keys kernel, low and high digit passes "
                             "over all jobs; the job table with the views stays resident, uploaded by "
                             "ws_plan_set_views)",
                   "parallelism": f"each of {world} ranks sorts its own 64-job batch, no collective"
                   if world > 1 else "single GPU",
                   "tuned": {str(b): {"tile": t, "ctas_per_sm": c, "segs_per_cta": g, "algorithm": ALGORITHMS[a]}
                             for b, (t, c, g, a) in tuned.items()}},
        "e2e": {"value": e2e_value, "unit": "Msplats/s", "h2d_bytes_per_step": pipe_h2d // pipe_steps,
                "d2h_bytes_per_step": pipe_d2h // pipe_steps,
                "call": "ws_sort_batch_host (one launch for all 64 jobs, then every job's survivor count and order "
                        "into pinned host buffers: the reference's outputs; its keys are never read back), from two "
                        "host threads with a context and stream each, steps alternating, so that one step's copy "
                        "to the host overlaps the next step's sort; wall time of all steps",
                "single_stream": {"value": e2e_single, "h2d_bytes_per_step": h2d // e2e_steps,
                                  "d2h_bytes_per_step": d2h // e2e_steps,
                                  "call": "the same call, one context, one step at a time (CUDA events around "
                                          "each step, which includes the call's host work)"}},
        "gpu_launches": 3 * args.steps,
        "clocks": clk,
    }
    if rank == 0:
        peak, src = peak_hbm()
        algo = sum(algorithmic_bytes(sp.count, s) for sp, s in zip(p["clouds"], survivors))
        achieved = algo / kernel_s / 1e9
        line["roofline"] = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                            "frac": achieved / peak, "traffic": ncu_traffic("mixed-64", args.cull),
                            "peak_source": src,
                            "kernel": "wsort::keys_kernel + digit_kernel<0> + digit_kernel<1>, one batched launch",
                            "kernel_us_per_step": kernel_s * 1e6, "algorithmic_bytes_per_step": algo,
                            "algorithmic_bytes": "32 N + 8 S summed over the jobs"}
        # the same 64 jobs as 64 plain calls
        time_plain(ctx, torch, p, reps, 2, flush)
        plain_rate = total * reps / (p["ms"] / 1e3) / 1e6
        graph_rate = value / world
        batch_rate = total * reps / (b_ms / 1e3) / 1e6
        line["cull0"] = cull0_batch(ctx, torch, p, flush, peak)
        line["batch"] = {"plain_msplats_s": plain_rate, "batch_call_msplats_s": batch_rate,
                         "graph_msplats_s": graph_rate, "graph_vs_plain": graph_rate / plain_rate,
                         "batch_call_vs_plain": batch_rate / plain_rate,
                         "plain_ms_per_step": p["ms"] / reps, "graph_ms_per_step": ms_max / args.steps,
                         "plain": "64 ws_sort calls (device outputs), each its own launch"}
    for sp in p["clouds"]:
        sp.destroy()
    return line, jobs


def pipelined_e2e(ctx, torch, jobs, p, tuned, steps, threads=2):
    """ws_sort_batch_host over the 64 jobs, `steps` calls from `threads` host
    threads, each with its own context and stream (each further context holds
    its own resident copy of the clouds and the same tuning). Returns (wall ms
    from the first call to the last result, host-to-device and device-to-host
    bytes of all calls)."""
    import ctypes
    import threading
    from winding_b200 import Context, autotune
    from winding_b200._lib import WsJob
    extra = []
    try:
        pairs = [(ctx, p)]
        for _ in range(threads - 1):
            c2 = Context(ctx.device)
            extra.append((c2, None))
            autotune.install(c2, tuned)
            q2 = load_jobs(c2, torch, jobs)
            extra[-1] = (c2, q2)
            pairs.append((c2, q2))
        sides = []
        for c, q in pairs:
            host = [(torch.empty(max(sp.count, 1), dtype=torch.int32).pin_memory(),
                     torch.zeros(1, dtype=torch.int32).pin_memory()) for sp in q["clouds"]]
            arr = (WsJob * len(host))()
            for j, (sp, v, (ho, hc)) in enumerate(zip(q["clouds"], q["views"], host)):
                arr[j].cloud, arr[j].view, arr[j].order, arr[j].keys, arr[j].count = (
                    sp.handle, v, ho.data_ptr(), None, hc.data_ptr())
            sides.append((c, arr, host, torch.cuda.Stream()))

        def run(side, n):
            c, arr, _, st = side
            for _ in range(n):
                c.check(c.lib.ws_sort_batch_host(c.handle, len(arr), arr, ctypes.c_void_p(st.cuda_stream)))

        for side in sides:
            run(side, 2)
        torch.cuda.synchronize()
        for c, *_ in sides:
            c.copy_stats(reset=True)
        t0 = time.perf_counter()
        workers = [threading.Thread(target=run, args=(side, steps // threads)) for side in sides]
        for th in workers:
            th.start()
        for th in workers:
            th.join()
        torch.cuda.synchronize()
        ms = (time.perf_counter() - t0) * 1e3
        h2d = d2h = 0
        for c, *_ in sides:
            a, b = c.copy_stats(reset=True)
            h2d, d2h = h2d + a, d2h + b
        want = [int(cc.item()) for _, _, cc in p["outs"]]
        for _, _, host, _ in sides:
            assert [int(hc[0]) for _, hc in host] == want
    finally:
        for c2, q2 in extra:
            if q2:
                for sp in q2["clouds"]:
                    sp.destroy()
            c2.close()
    return ms, h2d, d2h


def cull0_batch(ctx, torch, p, flush, peak, reps=5):
    """The same jobs at cull 0 (no footprint cull), as one ws_sort_batch
    launch: its kernels' event time, rate and roofline fraction."""
    from winding_b200 import make_view
    stream = torch.cuda.current_stream().cuda_stream
    views0 = [make_view(np.ctypeslib.as_array(v.model_view), np.ctypeslib.as_array(v.projection),
                        (v.viewport[0], v.viewport[1]), 0.0) for v in p["views"]]
    specs = [(sp, v0, o.data_ptr(), k.data_ptr(), c.data_ptr())
             for sp, v0, (o, k, c) in zip(p["clouds"], views0, p["outs"])]
    for _ in range(2):
        ctx.sort_batch(specs, stream)
    ctx.timing(True)
    timed_sorts(ctx, torch, reps, flush, lambda: ctx.sort_batch(specs, stream))
    kms, launches = ctx.timing_read()
    ctx.timing(False)
    ctx.sync()
    kernel_s = kms / max(launches, 1) / 1e3
    survivors = [int(c.item()) for _, _, c in p["outs"]]
    algo = sum(algorithmic_bytes(sp.count, s) for sp, s in zip(p["clouds"], survivors))
    return {"kernel_us": kernel_s * 1e6, "msplats_s": p["splats"] / kernel_s / 1e6, "survivors": sum(survivors),
            "achieved_gbs": algo / kernel_s / 1e9, "frac": algo / kernel_s / 1e9 / peak,
            "launch": "ws_sort_batch, kernels only (events)"}


def local_rank_of(torch):
    return torch.cuda.current_device()


def single_line(args, rank, world, dist, ctx, torch, flush):
    """One cloud (clusters-1M, uniform-100k or slab-6M): one plain ws_sort a
    step, one replica per rank."""
    jobs = make_jobs(args.workload, args.cull, seed_offset=0)
    p = load_jobs(ctx, torch, jobs)
    time_plain(ctx, torch, p, 0, args.warmup, flush)
    tuned = tune_batch(ctx, p, args)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local_rank_of(torch))
    clocks.start()
    time_plain(ctx, torch, p, args.steps, 0, flush)
    clk = clocks.stop()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ms_max = max_over_ranks(dist, torch, p["ms"])
    splats = p["splats"]
    value = splats * world * args.steps / (ms_max / 1e3) / 1e6
    survivors = p["survivors"]
    kms, launches = p["kernel_ms"], p["launches"]

    e2e_value, h2d, d2h, e2e_steps = single_e2e(ctx, torch, p, args.steps, flush)
    e2e_ms = max_over_ranks(dist, torch, splats * e2e_steps / e2e_value / 1e3)
    e2e_value = splats * world * e2e_steps / (e2e_ms / 1e3) / 1e6
    line = {
        "metric": "Msplats/s sorted (bit-exact stable order)", "value": value, "unit": "Msplats/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 keys, u32 sort", "data": "synthetic (seeded)",
        "config": {"workload": args.workload, "splats_per_step": splats * world,
                   "survivors_per_step": sum(survivors), "cull": args.cull, "viewport": [1920, 1080],
                   "l2": "flushed (256 MiB write) before each step",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "tuned": {str(b): {"tile": t, "ctas_per_sm": c, "segs_per_cta": g, "algorithm": ALGORITHMS[a]}
                             for b, (t, c, g, a) in tuned.items()}},
        "e2e": {"value": e2e_value, "unit": "Msplats/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "call": "ws_sort(WS_HOST_OUTPUT) into a pinned host buffer: the order and the survivor count, "
                        "the reference's outputs (its keys stay unsorted on the device and are never read back)"},
        # a lone job's ws_sort: the staging kernel, the keys kernel, two digit passes
        "gpu_launches": 4 * launches,
        "clocks": clk,
    }
    if rank == 0:
        peak, src = peak_hbm()
        front = survivors_at_cull0(ctx, torch, p) if args.cull > 0 else survivors
        algo = sum(algorithmic_bytes(sp.count, s) for sp, s in zip(p["clouds"], survivors))
        lay = sum(layout_bytes(sp.count, f, s, args.cull) for sp, f, s in zip(p["clouds"], front, survivors))
        kernel_s = kms / max(launches, 1) / 1e3
        achieved = algo / kernel_s / 1e9
        line["roofline"] = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                            "frac": achieved / peak, "traffic": ncu_traffic(args.workload, args.cull),
                            "peak_source": src, "kernel": "wsort::keys_kernel + digit_kernel<0> + digit_kernel<1>",
                            "kernel_us_per_step": kernel_s * 1e6, "algorithmic_bytes_per_step": algo,
                            "algorithmic_bytes": "32 N + 8 S", "layout_bytes_per_step": lay,
                            "layout_frac": lay / kernel_s / 1e9 / peak}
    for sp in p["clouds"]:
        sp.destroy()
    return line, jobs


def single_e2e(ctx, torch, p, steps, flush):
    """ws_sort with host outputs (the order and the count into a pinned
    buffer) per step: (Msplats/s, h2d and d2h bytes a step, steps)."""
    import ctypes
    from winding_b200 import _lib
    stream = torch.cuda.current_stream().cuda_stream
    n_max = max(sp.count for sp in p["clouds"])
    host_order = torch.empty(max(n_max, 1), dtype=torch.int32).pin_memory()
    cnt = ctypes.c_uint32()

    def one():
        for sp, v in zip(p["clouds"], p["views"]):
            ctx.check(ctx.lib.ws_sort(ctx.handle, sp.handle, ctypes.byref(v), host_order.data_ptr(),
                                      None, ctypes.byref(cnt), _lib.WS_HOST_OUTPUT, stream))

    for _ in range(2):
        one()
    e2e_steps = max(3, min(steps, 20))
    ctx.copy_stats(reset=True)
    ms = timed_sorts(ctx, torch, e2e_steps, flush, one, host_start=True)
    h2d, d2h = ctx.copy_stats(reset=True)
    return p["splats"] * e2e_steps / (ms / 1e3) / 1e6, h2d // e2e_steps, d2h // e2e_steps, e2e_steps


def suite(ctx, torch, flush, args):
    """Side measurements: the single-cloud sorts (clusters-1M, slab-6M)
    against the HBM roofline with their end-to-end rates, mixed-64 batched vs
    plain when it is not the headline, the served stream, particles,
    shading, decoding and drawing."""
    out = {}
    peak, src = peak_hbm()
    for name in ("clusters-1M", "slab-6M"):
        if name == args.workload:
            continue
        p = load_jobs(ctx, torch, make_jobs(name, 0.5))
        time_plain(ctx, torch, p, 0, 2, flush)
        tuned = tune_batch(ctx, p, argparse.Namespace(tile=0, ctas=0, segs=1))
        time_plain(ctx, torch, p, 20, 3, flush)
        n = p["splats"]
        algo = sum(algorithmic_bytes(sp.count, s) for sp, s in zip(p["clouds"], p["survivors"]))
        kernel_s = p["kernel_ms"] / p["launches"] / 1e3
        e2e, h2d, d2h, _ = single_e2e(ctx, torch, p, 20, flush)
        c0 = cull0_batch(ctx, torch, p, flush, peak)
        out[name] = {"cull0": c0, "splats": n, "survivors": p["survivors"][0], "kernel_us": kernel_s * 1e6,
                     "step_us": p["ms"] / 20 * 1e3, "msplats_s": n / (p["ms"] / 20 / 1e3) / 1e6,
                     "achieved_gbs": algo / kernel_s / 1e9, "frac": algo / kernel_s / 1e9 / peak,
                     "peak_source": src, "traffic": ncu_traffic(name, 0.5),
                     "e2e_msplats_s": e2e, "e2e_h2d_bytes": h2d, "e2e_d2h_bytes": d2h,
                     "tuned": {str(b): list(v) for b, v in tuned.items()}}
        for sp in p["clouds"]:
            sp.destroy()
        del p
    if args.workload != "mixed-64":
        line, _ = batch_line(argparse.Namespace(cull=0.5, warmup=3, steps=10, tile=0, ctas=0, segs=1), 0, 1, None,
                             ctx, torch, flush)
        out["mixed-64"] = {"graph_msplats_s": line["value"], "e2e_msplats_s": line["e2e"]["value"],
                           "frac": line["roofline"]["frac"], **line["batch"]}
    try:
        out["served-16"] = served(ctx, args)
    except Exception as exc:
        out["served-16"] = {"error": f"{type(exc).__name__}: {exc}"}
    for name, fn in (("particles-64", particles_suite), ("shade-1M", shade_suite), ("decode", decode_suite),
                     ("draw-1M", draw_suite)):
        try:
            out[name] = fn(ctx, torch, flush, peak)
        except Exception as exc:
            out[name] = {"error": f"{type(exc).__name__}: {exc}"}
    return out


def particles_suite(ctx, torch, flush, peak):
    """64 alpha emitters of 1k-200k particles in one pool: one batched launch
    (ws_sort_particles over all) against one launch per emitter, as the
    reference dispatches them (render/particles.js:838-850)."""
    from winding_b200 import particles as P, workloads as W
    rings = W.emitter_rings()
    n = sum(c for _, c in rings)
    pool = torch.from_numpy(W.particle_pool(n).reshape(-1)).cuda()
    eye = np.array([0.0, 5.0, 80.0], np.float32)
    fwd = np.array([0.0, -0.0624, -0.998], np.float32)
    outs = [(torch.empty(max(c, 1), dtype=torch.int32, device="cuda"), torch.empty(max(c, 1), dtype=torch.int32,
             device="cuda"), torch.zeros(1, dtype=torch.int32, device="cuda")) for _, c in rings]
    ptrs = [(o.data_ptr(), k.data_ptr(), c.data_ptr()) for o, k, c in outs]
    stream = torch.cuda.current_stream().cuda_stream

    def batched():
        P.sort_emitters(ctx, pool.data_ptr(), rings, eye, fwd, ptrs, stream)

    def plain():
        for ring, out in zip(rings, ptrs):
            P.sort_emitters(ctx, pool.data_ptr(), [ring], eye, fwd, [out], stream)

    for _ in range(3):
        batched()
        plain()
    ctx.timing(True)
    b_ms = timed_sorts(ctx, torch, 10, flush, batched)
    kms, launches = ctx.timing_read()
    ctx.timing(False)
    p_ms = timed_sorts(ctx, torch, 10, flush, plain)
    live = sum(int(c.item()) for _, _, c in outs)
    kernel_s = kms / max(launches, 1) / 1e3
    algo = 32 * n + 8 * live
    return {"emitters": len(rings), "particles": n, "live": live,
            "batched_mparticles_s": n * 10 / (b_ms / 1e3) / 1e6, "plain_mparticles_s": n * 10 / (p_ms / 1e3) / 1e6,
            "batched_vs_plain": p_ms / b_ms, "kernel_us": kernel_s * 1e6,
            "achieved_gbs": algo / kernel_s / 1e9, "frac": algo / kernel_s / 1e9 / peak,
            "algorithmic_bytes": "32 per slot + 8 per live particle"}


def shade_suite(ctx, torch, flush, peak):
    """clusters-1M with degree-3 harmonics: the sort alone against the sort
    with the shade pass fused into it (ws_sort_batch_shaded)."""
    from winding_b200 import parse_splats, workloads as W
    from winding_b200.splats import eye_in_cloud
    job = W.clusters_1m(seed=1, cull=0.5)
    sp = parse_splats(job.records, ctx)
    sp.set_harmonics(3, W.harmonics_words(sp.count, 3))
    from winding_b200 import make_view
    view = make_view(job.view.model_view, job.view.projection, job.view.viewport, 0.5)
    o = torch.empty(sp.count, dtype=torch.int32, device="cuda")
    k = torch.empty_like(o)
    c = torch.zeros(1, dtype=torch.int32, device="cuda")
    shaded = torch.empty_like(o)
    spec = [(sp, view, o.data_ptr(), k.data_ptr(), c.data_ptr())]
    shade = [(eye_in_cloud(job.view.model_view), shaded.data_ptr())]
    stream = torch.cuda.current_stream().cuda_stream
    res = {}
    for name, fn in (("sort", lambda: ctx.sort_batch(spec, stream)),
                     ("sort_and_shade", lambda: ctx.sort_batch_shaded(spec, shade, stream))):
        for _ in range(3):
            fn()
        ctx.timing(True)
        timed_sorts(ctx, torch, 10, flush, fn)
        kms, launches = ctx.timing_read()
        ctx.timing(False)
        res[name + "_kernel_us"] = kms / max(launches, 1) * 1e3
    s = int(c.item())
    extra_s = (res["sort_and_shade_kernel_us"] - res["sort_kernel_us"]) / 1e6
    res.update({"splats": sp.count, "survivors": s, "degree": 3,
                "shade_bytes": s * (23 * 4 + 4), "shade_extra_us": extra_s * 1e6,
                "shade_gbs": s * 96 / extra_s / 1e9 if extra_s > 0 else None})
    sp.destroy()
    return res


def draw_suite(ctx, torch, flush, peak):
    """clusters-1M sorted and drawn into a 1920 x 1080 RGBA f32 image
    (ws_draw): the draw alone, timed with CUDA events around the call (it
    synchronises its stream once, to size the binning)."""
    from winding_b200 import make_view, parse_splats, workloads as W
    job = W.clusters_1m(seed=1, cull=0.5)
    sp = parse_splats(job.records, ctx)
    view = make_view(job.view.model_view, job.view.projection, job.view.viewport, 0.5)
    o = torch.empty(sp.count, dtype=torch.int32, device="cuda")
    k = torch.empty_like(o)
    c = torch.zeros(1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    ctx.sort_device(sp, view, o.data_ptr(), k.data_ptr(), c.data_ptr(), stream)
    img = torch.zeros((1080, 1920, 4), dtype=torch.float32, device="cuda")

    def draw():
        img.zero_()
        ctx.draw(sp, view, o.data_ptr(), c.data_ptr(), img.data_ptr(), 1920, 1080, None, stream)

    for _ in range(3):
        draw()
    ms = timed_sorts(ctx, torch, 10, flush, draw) / 10
    drawn = int(c.item())
    covered = float((img[..., 3] > 0).float().mean().item())
    sp.destroy()
    return {"splats": 1_000_000, "drawn": drawn, "width": 1920, "height": 1080, "ms": ms,
            "msplats_s": drawn / (ms / 1e3) / 1e6, "covered_fraction": covered,
            "note": "includes clearing the 33 MB image and the call's one stream sync"}


def decode_suite(ctx, torch, flush, peak):
    """Loading a capture through the public call (ws_cloud_load): a 1M-splat
    .ply with degree-3 harmonics and 1M .splat records, host bytes to a
    resident cloud (header parse, upload, device decode)."""
    from winding_b200 import load_splats, workloads as W
    out = {}
    ply = W.ply_bytes(1_000_000, 3)
    rec = W.clusters(1_000_000, 1).tobytes()
    for name, data in (("ply_deg3", ply), ("splat", rec)):
        load_splats(data, ctx).destroy()
        times = []
        for _ in range(3):
            t0 = time.perf_counter()
            sp = load_splats(data, ctx)
            times.append(time.perf_counter() - t0)
            sp.destroy()
        t = min(times)
        out[name] = {"splats": 1_000_000, "bytes": len(data), "ms": t * 1e3, "msplats_s": 1.0 / t,
                     "gb_s": len(data) / t / 1e9}
    return out


def served(ctx, args, rates=(2000.0, 20000.0, 50000.0), seconds: float = 0.5, repeats: int = 5):
    """Config 4: Poisson streams of random-pose requests over 16 resident
    scenes of 50k-4M splats, through the server (continuous batching) and,
    on the same arrival schedule, through one plain ws_sort per request. Per
    arrival rate: one warm-up run, then `repeats` runs of `seconds` each,
    reported as the median with the spread (min, max). Then a saturated
    queue (every request submitted at once)."""
    import threading
    import ctypes as _ct
    import torch
    from winding_b200 import make_view, parse_splats, workloads as W
    from winding_b200.server import Server
    scenes = [parse_splats(rec, ctx) for rec in W.served_16()]
    resident = sum(sp.count for sp in scenes) * 40
    proj = W.perspective(W.FOV_Y, W.ASPECT, W.NEAR)

    def requests(rate, dur, seed):
        arrivals = W.poisson_arrivals(rate, dur, seed=seed)
        rng = np.random.default_rng(seed + 1)
        reqs = [(int(rng.integers(0, len(scenes))), make_view(W.random_pose(rng), proj, W.VIEWPORT, 0.5))
                for _ in arrivals]
        return arrivals, reqs

    def run(arrivals, reqs, submit, collect):
        """Submits on the arrival schedule from one thread, collects from another;
        returns (seconds from the first arrival to the last result, latencies in
        ms from each request's scheduled arrival to its result)."""
        done = [None] * len(reqs)
        tickets = [None] * len(reqs)
        ready = threading.Semaphore(0)
        t0 = time.perf_counter()

        def producer():
            for k, (at, (sc, v)) in enumerate(zip(arrivals, reqs)):
                delay = t0 + at - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
                tickets[k] = (t0 + at, submit(scenes[sc], v))
                ready.release()

        th = threading.Thread(target=producer)
        th.start()
        for k in range(len(reqs)):
            ready.acquire()
            t_sub, tk = tickets[k]
            collect(tk)
            done[k] = (time.perf_counter() - t_sub) * 1e3
        th.join()
        return time.perf_counter() - t0, done

    def collect(srv, t):
        srv.result(t)      # the result is on the device, as the reference's draw reads it
        srv.release(t)

    n_max = max(sp.count for sp in scenes)
    o = torch.empty(n_max, dtype=torch.int32, device="cuda")
    k = torch.empty(n_max, dtype=torch.int32, device="cuda")
    c = torch.zeros(1, dtype=torch.int32, device="cuda")
    cnt = _ct.c_uint32()

    def plain(sp, v):
        """One plain ws_sort per request, device outputs, then its count."""
        ctx.sort_device(sp, v, o.data_ptr(), k.data_ptr(), c.data_ptr())
        ctx.check(ctx.lib.ws_device_download(ctx.handle, c.data_ptr(), _ct.byref(cnt), 4, None))

    def spread(vals):
        return {"median": float(np.median(vals)), "min": float(np.min(vals)), "max": float(np.max(vals))}

    out = {"scenes": len(scenes), "resident_bytes": resident, "seconds_per_run": seconds, "repeats": repeats,
           "latency": "scheduled arrival to the result ready in device memory, count known on the host"}
    with Server(ctx, memory_budget=8 << 30, max_batch=64, streams=2) as srv:
        for rate in rates:
            warm_a, warm_r = requests(rate, 0.1, 99)
            run(warm_a, warm_r, lambda sp, v: srv.submit(sp, v), lambda t: collect(srv, t))
            run(warm_a, warm_r, plain, lambda res: None)
            s_rate, s_p50, s_p99, s_batch, p_rate, p_p50, p_p99, n_req = [], [], [], [], [], [], [], []
            for r in range(repeats):
                arrivals, reqs = requests(rate, seconds, 5 + 17 * r)
                splats = sum(scenes[q].count for q, _ in reqs)
                before = srv.stats()
                wall, lat = run(arrivals, reqs, lambda sp, v: srv.submit(sp, v), lambda t: collect(srv, t))
                after = srv.stats()
                batches = after["batches"] - before["batches"]
                s_rate.append(splats / wall / 1e6)
                s_p50.append(float(np.percentile(lat, 50)))
                s_p99.append(float(np.percentile(lat, 99)))
                s_batch.append(len(reqs) / max(batches, 1))
                wall, lat = run(arrivals, reqs, plain, lambda res: None)
                p_rate.append(splats / wall / 1e6)
                p_p50.append(float(np.percentile(lat, 50)))
                p_p99.append(float(np.percentile(lat, 99)))
                n_req.append(len(reqs))
            out[f"{int(rate)}hz"] = {
                "requests_per_run": spread(n_req), "served_msplats_s": spread(s_rate),
                "served_p50_ms": spread(s_p50), "served_p99_ms": spread(s_p99), "mean_batch": spread(s_batch),
                "plain_msplats_s": spread(p_rate), "plain_p50_ms": spread(p_p50), "plain_p99_ms": spread(p_p99),
                "served_vs_plain": float(np.median(s_rate) / np.median(p_rate))}
        st = srv.stats()
        out["overlapped_batches"] = st["overlapped_batches"]
        out["admission_waits"] = st["admission_waits"]
        out["device_p50_ms"] = st["p50_ms"]
        out["device_p99_ms"] = st["p99_ms"]

    # Saturated: every request queued at once (a closed queue), so the server
    # batches as many as it admits; against one plain sort per request.
    _, burst = requests(20000.0, 0.06, 7)
    burst = burst[:1024]
    burst_splats = sum(scenes[q].count for q, _ in burst)
    sat_s, sat_p, sat_b = [], [], []
    with Server(ctx, memory_budget=8 << 30, max_batch=64, streams=2) as srv:
        for r in range(repeats + 1):
            before = srv.stats()
            t0 = time.perf_counter()
            tickets = [srv.submit(scenes[sc], v) for sc, v in burst]
            for tk in tickets:
                collect(srv, tk)
            wall = time.perf_counter() - t0
            after = srv.stats()
            t0 = time.perf_counter()
            for sc, v in burst:
                plain(scenes[sc], v)
            p_wall = time.perf_counter() - t0
            if r:   # the first round is the warm-up
                sat_s.append(burst_splats / wall / 1e6)
                sat_p.append(burst_splats / p_wall / 1e6)
                sat_b.append(len(burst) / max(after["batches"] - before["batches"], 1))
    out["saturated"] = {"requests": len(burst), "splats": burst_splats, "served_msplats_s": spread(sat_s),
                        "plain_msplats_s": spread(sat_p), "mean_batch": spread(sat_b),
                        "served_vs_plain": float(np.median(sat_s) / np.median(sat_p))}
    for sp in scenes:
        sp.destroy()
    return out


def main():
    args = parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        run_wsort(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
