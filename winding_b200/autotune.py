"""The sort's autotuner: algorithm, kernel variant and segment sizing per
launch size.

A candidate is (tile, ctas_per_sm, segs_per_cta, algorithm). Algorithm 0
sorts in three phases (keys, then two 8-bit digit passes) over segments of
every job: tile is the least splats a segment covers, ctas_per_sm the digit
passes' kernel variant (1: CTAs of 1024 threads, one an SM; 2: CTAs of 512
threads, two an SM) and segs_per_cta the segments cut per resident CTA.
Algorithms 1 and 2 give each job one CTA that sorts it in shared memory in
one kernel, with two 8-bit passes (radix) or one counting pass over all
65536 keys; they are candidates when every job of the workload has at most
16384 splats. For a workload (or synthetic clouds of given sizes) every
candidate is timed with
the library's own CUDA-event kernel timing (ws_timing) over a few launches,
and the fastest is installed in the context's tuning table for that launch
size (floor(log2(total splats)), ws_set_tuning). Results persist in a JSON
cache keyed by the GPU's name, so later processes load them instead of
measuring.

    table = autotune.tune(ctx, [[(splats, view)]], cache="~/.cache/wsort_tuning.json")
"""
from __future__ import annotations

import json
import os

from . import _lib

TILES = (1024, 2048, 8192)
CTAS = (1, 2)
SEGS = (1, 2, 4)
CANDIDATES = tuple((t, c, s, _lib.ALGO_PHASES) for t in TILES for c in CTAS for s in SEGS)
ONE_CTA_CANDIDATES = ((2048, 1, 1, _lib.ALGO_ONE_RADIX), (2048, 1, 1, _lib.ALGO_ONE_COUNT))


def bucket(splats: int) -> int:
    return max(int(splats).bit_length() - 1, 0)


def gpu_name(device: int = 0) -> str:
    try:
        import torch
        return torch.cuda.get_device_name(device)
    except Exception:
        return f"device{device}"


def _time_jobs(ctx, jobs, reps: int) -> float:
    """Mean sort-kernel ms of one batched launch of `jobs` (device outputs)."""
    import torch
    specs = []
    keep = []
    for sp, view in jobs:
        n = max(sp.count, 1)
        o = torch.empty(n, dtype=torch.int32, device="cuda")
        k = torch.empty(n, dtype=torch.int32, device="cuda")
        c = torch.zeros(1, dtype=torch.int32, device="cuda")
        keep += [o, k, c]
        specs.append((sp, view, o.data_ptr(), k.data_ptr(), c.data_ptr()))
    stream = torch.cuda.current_stream().cuda_stream
    ctx.sort_batch(specs, stream)
    torch.cuda.synchronize()
    ctx.timing(True)
    for _ in range(reps):
        ctx.sort_batch(specs, stream)
    ms, n = ctx.timing_read()
    ctx.timing(False)
    ctx.sync()
    return ms / max(n, 1)


def candidates_for(jobs, candidates=CANDIDATES) -> tuple:
    """The candidates for a batch: the one-CTA sorts too when every job is
    small enough for them."""
    if jobs and all(sp.count <= _lib.ONE_CTA_MAX for sp, _ in jobs):
        return tuple(candidates) + ONE_CTA_CANDIDATES
    return tuple(candidates)


def measure(ctx, jobs, reps: int = 5, candidates=CANDIDATES) -> list[tuple[float, tuple[int, int, int, int]]]:
    """(ms, candidate) for every candidate on one batch of jobs, fastest first."""
    saved = ctx.params
    table_off = (_lib.WsParams * 1)()
    ctx.check(ctx.lib.ws_set_tuning(ctx.handle, table_off, 0))
    out = []
    try:
        for cand in candidates:
            tile, ctas, segs, algorithm = _full(cand)
            ctx.set_params(tile=tile, ctas_per_sm=ctas, segs_per_cta=segs, algorithm=algorithm)
            out.append((_time_jobs(ctx, jobs, reps), _full(cand)))
    finally:
        ctx.set_params(tile=saved.tile, ctas_per_sm=saved.ctas_per_sm, segs_per_cta=saved.segs_per_cta,
                       algorithm=saved.algorithm)
    return sorted(out)


def install(ctx, table: dict[int, tuple]) -> None:
    """Installs {bucket: (tile, ctas, segs[, algorithm])} as the context's tuning table."""
    n = max(table) + 1 if table else 0
    arr = (_lib.WsParams * max(n, 1))()
    spin = ctx.params.spin_limit
    for b, cand in table.items():
        arr[b].tile, arr[b].ctas_per_sm, arr[b].segs_per_cta, arr[b].algorithm = _full(cand)
        arr[b].spin_limit = spin
    ctx.check(ctx.lib.ws_set_tuning(ctx.handle, arr, n))


def _full(v) -> tuple[int, int, int, int]:
    """A candidate with its algorithm (0 when an older cache left it out)."""
    v = tuple(int(x) for x in v)
    return v if len(v) == 4 else v + (_lib.ALGO_PHASES,)


def _valid(v) -> bool:
    return isinstance(v, (list, tuple)) and len(v) in (3, 4) and tuple(v[:1]) != (0,)


def tune(ctx, workloads, cache: str | None = None, reps: int = 5, force: bool = False,
         candidates=CANDIDATES) -> dict[int, tuple[int, int, int, int]]:
    """workloads: batches, each a list of (splats, view). Measures each (unless
    its size bucket is in the cache), installs the table and returns it."""
    key = gpu_name(ctx.device)
    stored: dict = {}
    if cache and os.path.exists(os.path.expanduser(cache)):
        try:
            with open(os.path.expanduser(cache)) as f:
                stored = json.load(f)
        except (OSError, ValueError):
            stored = {}
    table = {int(b): _full(v) for b, v in stored.get(key, {}).items() if _valid(v)}
    for jobs in workloads:
        b = bucket(sum(sp.count for sp, _ in jobs))
        if b in table and not force:
            continue
        table[b] = measure(ctx, jobs, reps, candidates_for(jobs, candidates))[0][1]
    install(ctx, table)
    if cache:
        stored[key] = {str(b): list(v) for b, v in sorted(table.items())}
        path = os.path.expanduser(cache)
        os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
        with open(path, "w") as f:
            json.dump(stored, f, indent=1)
    return table


def load(ctx, cache: str) -> dict[int, tuple[int, int, int, int]]:
    """Installs a cached table for this GPU, if there is one."""
    path = os.path.expanduser(cache)
    if not os.path.exists(path):
        return {}
    with open(path) as f:
        stored = json.load(f)
    table = {int(b): _full(v) for b, v in stored.get(gpu_name(ctx.device), {}).items() if _valid(v)}
    if table:
        install(ctx, table)
    return table
