"""ws_sort_noalloc, the sort entry point that allocates no device memory.

Some callers cannot allocate when they sort: a plugin whose device memory
belongs to the host application's pool, or a frame loop that may not stall on
cudaMalloc / cudaFree. For them ws_sort_noalloc runs the same sort on a fixed
scratch array inside the library. These tests call it through the C ABI and
check its output against the oracle and against ws_sort (the existing entry
point), two calls in a row (the second shares the scratch the first left
behind), from one splat to the largest cloud it takes; then that a run of its
calls allocates nothing (the device's free memory is unchanged, and the
library's own buffer growths, made to fail, are never attempted). The file is
collected last, and passes both alone in a fresh process and after the other
tests.
"""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O
from winding_b200 import _lib, make_view, parse_splats, workloads as W

pytestmark = pytest.mark.gpu


def _noalloc(ctx, splats, view, torch):
    n = max(splats.count, 1)
    stream = torch.cuda.current_stream().cuda_stream
    order = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    keys = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    count = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = ctx.lib.ws_sort_noalloc(splats.handle, ctypes.byref(view), order.data_ptr(), keys.data_ptr(),
                                 count.data_ptr(), stream)
    assert rc == _lib.WS_OK, rc
    torch.cuda.synchronize()
    s = int(count.item())
    assert s != -1, "ws_sort_noalloc: a device-side wait gave up"
    return order[:s].cpu().numpy().view(np.uint32), keys[:s].cpu().numpy().view(np.uint32)


CASES = [
    ("clusters", 700_000, 0.5),
    ("slab", 900_000, 0.0),
    ("uniform", 100_000, 0.5),
    ("uniform", 1, 0.5),
    ("uniform", _lib.WS_NOALLOC_MAX_SPLATS, 0.5),
]


@pytest.mark.parametrize("kind,n,cull", CASES)
def test_noalloc_matches_the_oracle_and_ws_sort(ctx, kind, n, cull):
    import torch
    job = {"clusters": lambda: W.clusters_1m(seed=61, n=n), "slab": lambda: W.slab_6m(seed=62, n=n),
           "uniform": lambda: W.uniform_100k(seed=64 + n % 7, n=n)}[kind]()
    splats = parse_splats(job.records, ctx)
    try:
        view = make_view(job.view.model_view, job.view.projection, job.view.viewport, cull)
        want_o, want_k = O.sort_view(O.parse_splat(job.bytes()), job.view.model_view, job.view.projection,
                                     job.view.viewport, cull)
        for _ in range(2):
            order, keys = _noalloc(ctx, splats, view, torch)
            assert np.array_equal(order, want_o) and np.array_equal(keys, want_k)
        got_o, got_k = ctx.sort(splats, view)
        assert np.array_equal(got_o, want_o) and np.array_equal(got_k, want_k)
    finally:
        splats.destroy()


def test_noalloc_allocates_nothing(ctx):
    import torch
    jobs = [W.uniform_100k(seed=70 + k, n=n) for k, n in enumerate((1, 5000, 300_000, _lib.WS_NOALLOC_MAX_SPLATS))]
    clouds = [parse_splats(j.records, ctx) for j in jobs]
    views = [make_view(j.view.model_view, j.view.projection, j.view.viewport, 0.5) for j in jobs]
    n = _lib.WS_NOALLOC_MAX_SPLATS
    order = torch.empty(n, dtype=torch.int32, device="cuda")
    keys = torch.empty(n, dtype=torch.int32, device="cuda")
    count = torch.zeros(1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream

    def call(sp, v):
        return ctx.lib.ws_sort_noalloc(sp.handle, ctypes.byref(v), order.data_ptr(), keys.data_ptr(),
                                       count.data_ptr(), stream)

    try:
        assert call(clouds[0], views[0]) == _lib.WS_OK   # the first call on the device takes the array's address
        torch.cuda.synchronize()
        free_before, _ = torch.cuda.mem_get_info()
        _lib.load().ws_inject_alloc_failures(1000)
        for _ in range(2):
            for sp, v in zip(clouds, views):
                assert call(sp, v) == _lib.WS_OK
        torch.cuda.synchronize()
        free_after, _ = torch.cuda.mem_get_info()
        assert free_after == free_before
        assert int(count.item()) != -1
    finally:
        _lib.load().ws_inject_alloc_failures(0)
        for sp in clouds:
            sp.destroy()


def test_noalloc_wait_that_runs_out_sets_the_count_and_the_next_call_is_exact(ctx):
    """A job on the fixed array whose first phase is left out: its bounded
    wait gives up, the closing check turns that into *count = 0xFFFFFFFF, and
    the next ws_sort_noalloc on the same array is exact again."""
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    count = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert ctx.lib.ws_selftest_noalloc_wait(ctx.handle, 0, count.data_ptr(), stream) == _lib.WS_ERR_ARG
    assert ctx.lib.ws_selftest_noalloc_wait(ctx.handle, 2000, count.data_ptr(), stream) == _lib.WS_OK
    torch.cuda.synchronize()
    assert int(count.item()) == -1
    job = W.clusters_1m(seed=65, n=120_000)
    splats = parse_splats(job.records, ctx)
    try:
        view = make_view(job.view.model_view, job.view.projection, job.view.viewport, 0.5)
        want_o, want_k = O.sort_view(O.parse_splat(job.bytes()), job.view.model_view, job.view.projection,
                                     job.view.viewport, 0.5)
        order, keys = _noalloc(ctx, splats, view, torch)
        assert np.array_equal(order, want_o) and np.array_equal(keys, want_k)
    finally:
        splats.destroy()


def test_noalloc_refuses_clouds_beyond_its_fixed_size(ctx):
    import torch
    job = W.uniform_100k(seed=63, n=_lib.WS_NOALLOC_MAX_SPLATS + 1)
    splats = parse_splats(job.records, ctx)
    view = make_view(job.view.model_view, job.view.projection, job.view.viewport, 0.5)
    out = torch.empty(splats.count, dtype=torch.int32, device="cuda")
    count = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = ctx.lib.ws_sort_noalloc(splats.handle, ctypes.byref(view), out.data_ptr(), None, count.data_ptr(), None)
    assert rc == _lib.WS_ERR_CAPACITY
    splats.destroy()
