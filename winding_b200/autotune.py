"""The sort's autotuner: tile size and kernel variant per launch size.

For a workload (or synthetic clouds of given sizes), every candidate
(tile 1024 / 2048 / 4096 x 2 / 3 / 4 resident CTAs per SM, and tile 1024 x 6)
is timed with the
library's own CUDA-event kernel timing (ws_timing) over a few launches, and
the fastest is installed in the context's tuning table for that launch size
(floor(log2(total splats)), ws_set_tuning). Results persist in a JSON cache
keyed by the GPU's name, so later processes load them instead of measuring.

    table = autotune.tune(ctx, [(splats, view)], cache="~/.cache/wsort_tuning.json")
"""
from __future__ import annotations

import json
import os

from . import _lib

TILES = (1024, 2048, 4096)
CTAS = (2, 3, 4)
CANDIDATES = tuple((t, c) for t in TILES for c in CTAS) + ((1024, 6),)


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


def measure(ctx, jobs, reps: int = 5) -> list[tuple[float, int, int]]:
    """(ms, tile, ctas) for every candidate on one batch of jobs."""
    saved = ctx.params
    table_off = (_lib.WsParams * 1)()
    ctx.check(ctx.lib.ws_set_tuning(ctx.handle, table_off, 0))
    out = []
    try:
        for tile, ctas in CANDIDATES:
            ctx.set_params(tile=tile, ctas_per_sm=ctas)
            out.append((_time_jobs(ctx, jobs, reps), tile, ctas))
    finally:
        ctx.set_params(tile=saved.tile, ctas_per_sm=saved.ctas_per_sm)
    return sorted(out)


def install(ctx, table: dict[int, tuple[int, int]]) -> None:
    """Installs {bucket: (tile, ctas)} as the context's tuning table."""
    n = max(table) + 1 if table else 0
    arr = (_lib.WsParams * max(n, 1))()
    spin = ctx.params.spin_limit
    for b, (tile, ctas) in table.items():
        arr[b].tile = tile
        arr[b].ctas_per_sm = ctas
        arr[b].spin_limit = spin
    ctx.check(ctx.lib.ws_set_tuning(ctx.handle, arr, n))


def tune(ctx, workloads, cache: str | None = None, reps: int = 5, force: bool = False) -> dict[int, tuple[int, int]]:
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
    table = {int(b): tuple(v) for b, v in stored.get(key, {}).items()}
    for jobs in workloads:
        b = bucket(sum(sp.count for sp, _ in jobs))
        if b in table and not force:
            continue
        ms, tile, ctas = measure(ctx, jobs, reps)[0]
        table[b] = (tile, ctas)
    install(ctx, table)
    if cache:
        stored[key] = {str(b): list(v) for b, v in sorted(table.items())}
        path = os.path.expanduser(cache)
        os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
        with open(path, "w") as f:
            json.dump(stored, f, indent=1)
    return table


def load(ctx, cache: str) -> dict[int, tuple[int, int]]:
    """Installs a cached table for this GPU, if there is one."""
    path = os.path.expanduser(cache)
    if not os.path.exists(path):
        return {}
    with open(path) as f:
        stored = json.load(f)
    table = {int(b): tuple(v) for b, v in stored.get(gpu_name(ctx.device), {}).items()}
    if table:
        install(ctx, table)
    return table
