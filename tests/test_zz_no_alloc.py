"""ws_sort_noalloc, the sort entry point that allocates no device memory.

Some callers cannot allocate when they sort: a plugin whose device memory
belongs to the host application's pool, or a frame loop that may not stall on
cudaMalloc / cudaFree. For them ws_sort_noalloc runs the same sort on a fixed
scratch array inside the library. This test calls it through the C ABI and
checks its output against ws_sort's (the existing entry point) on two calls in
a row, exactly, as every parity test here does: the second call shares the
scratch the first one left behind. It sits in a file of its own, collected
last, and passes both alone in a fresh process and after the other tests.
"""
import ctypes

import numpy as np
import pytest

from winding_b200 import _lib, make_view, parse_splats, workloads as W

pytestmark = pytest.mark.gpu


def _sort_both(ctx, splats, view, torch):
    n = max(splats.count, 1)
    stream = torch.cuda.current_stream().cuda_stream
    outs = []
    for fn in ("ws_sort", "ws_sort_noalloc"):
        order = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        keys = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        count = torch.zeros(1, dtype=torch.int32, device="cuda")
        if fn == "ws_sort":
            rc = ctx.lib.ws_sort(ctx.handle, splats.handle, ctypes.byref(view), order.data_ptr(), keys.data_ptr(),
                                 count.data_ptr(), _lib.WS_DEVICE_OUTPUT, stream)
        else:
            rc = ctx.lib.ws_sort_noalloc(splats.handle, ctypes.byref(view), order.data_ptr(), keys.data_ptr(),
                                         count.data_ptr(), stream)
        assert rc == _lib.WS_OK, (fn, rc)
        torch.cuda.synchronize()
        s = int(count.item())
        assert s != -1, f"{fn}: a device-side wait gave up"
        outs.append((s, order[:s].cpu().numpy().view(np.uint32), keys[:s].cpu().numpy().view(np.uint32)))
    return outs


def test_noalloc_matches_ws_sort_twice_in_a_row(ctx):
    import torch
    jobs = [W.clusters_1m(seed=61, n=700_000), W.slab_6m(seed=62, n=900_000)]
    for job, cull in zip(jobs, (0.5, 0.0)):
        splats = parse_splats(job.records, ctx)
        view = make_view(job.view.model_view, job.view.projection, job.view.viewport, cull)
        (s0, o0, k0), (s1, o1, k1) = _sort_both(ctx, splats, view, torch)
        assert s0 == s1 and s0 > 0
        assert np.array_equal(o0, o1) and np.array_equal(k0, k1)
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
