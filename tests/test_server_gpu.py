"""The request loop: continuous batching over resident clouds.

Each result must be identical alone and in the mix (exactly: the sort is
integer work after pinned f32 keys), and equal to the oracle's.
"""
import threading

import numpy as np
import pytest

from oracle import oracle as O
from winding_b200 import make_view, parse_splats, workloads as W
from winding_b200.server import Server

pytestmark = pytest.mark.gpu


def _scenes(ctx, counts, seed):
    rng = np.random.default_rng(seed)
    out = []
    for j, n in enumerate(counts):
        rec = W.scene(W.KINDS[j % 3], n, seed * 100 + j)
        out.append((rec, parse_splats(rec, ctx), O.parse_splat(rec.tobytes())))
    return out, rng


def _view(rng, cull=0.5):
    return W.View(W.random_pose(rng), W.perspective(W.FOV_Y, W.ASPECT, W.NEAR), W.VIEWPORT, cull)


def test_each_result_is_the_same_alone_and_in_the_mix(ctx):
    scenes, rng = _scenes(ctx, [20_000, 150_000, 60_000, 400_000, 5_000], 7)
    reqs = [(s, _view(rng, 0.5 if k % 2 else 0.0)) for k in range(40) for s in [scenes[k % len(scenes)]]]
    with Server(ctx, memory_budget=1 << 30, max_batch=16) as srv:
        # alone: one request at a time
        alone = []
        for (rec, sp, parsed), v in reqs:
            t = srv.submit(sp, make_view(v.model_view, v.projection, v.viewport, v.cull))
            alone.append(srv.wait(t))
        # in the mix: everything at once, from two threads
        tickets = [None] * len(reqs)

        def submit(lo, hi):
            for k in range(lo, hi):
                (rec, sp, parsed), v = reqs[k]
                tickets[k] = srv.submit(sp, make_view(v.model_view, v.projection, v.viewport, v.cull))
        th = [threading.Thread(target=submit, args=(0, 20)), threading.Thread(target=submit, args=(20, 40))]
        for t in th:
            t.start()
        for t in th:
            t.join()
        mixed = [srv.wait(t) for t in tickets]
        st = srv.stats()
    assert st["completed"] == 80 and st["failed"] == 0
    assert st["max_batch_seen"] > 1          # the mix was batched
    for ((rec, sp, parsed), v), a, m in zip(reqs, alone, mixed):
        assert np.array_equal(a[0], m[0]) and np.array_equal(a[1], m[1])
        want_o, want_k = O.sort_view(parsed, v.model_view, v.projection, v.viewport, v.cull)
        assert np.array_equal(m[0], want_o) and np.array_equal(m[1], want_k)
    for _, sp, _ in scenes:
        sp.destroy()


def test_admission_by_memory(ctx):
    """A budget that holds two requests at a time: the rest wait for memory,
    and every result is still right."""
    scenes, rng = _scenes(ctx, [300_000, 300_000, 300_000], 8)
    budget = 2 * 300_000 * 17 + (2 << 20)
    views = [_view(rng) for _ in range(12)]
    with Server(ctx, memory_budget=budget, max_batch=8) as srv:
        tickets = [srv.submit(scenes[k % 3][1], make_view(v.model_view, v.projection, v.viewport, v.cull))
                   for k, v in enumerate(views)]
        results = [srv.wait(t) for t in tickets]
        st = srv.stats()
    assert st["completed"] == 12 and st["admission_waits"] > 0
    for k, (v, (order, keys)) in enumerate(zip(views, results)):
        parsed = scenes[k % 3][2]
        want_o, want_k = O.sort_view(parsed, v.model_view, v.projection, v.viewport, v.cull)
        assert np.array_equal(order, want_o) and np.array_equal(keys, want_k)
    for _, sp, _ in scenes:
        sp.destroy()


def test_refusals(ctx):
    from winding_b200 import WsError
    scenes, rng = _scenes(ctx, [100_000], 9)
    with Server(ctx, memory_budget=1 << 20) as srv:
        with pytest.raises(WsError, match="WS_ERR_NOMEM"):      # alone it exceeds the budget
            srv.submit(scenes[0][1], make_view(*_view(rng).__dict__.values()))
    with Server(ctx, memory_budget=1 << 28) as srv:
        v = _view(rng)
        with pytest.raises(WsError, match="WS_ERR_ARG"):
            srv.submit(scenes[0][1], make_view(v.model_view, v.projection, v.viewport, -1.0))
        scenes[0][1].destroy()
        with pytest.raises(WsError, match="WS_ERR_UNLOADED"):
            srv.submit(scenes[0][1], make_view(v.model_view, v.projection, v.viewport, 0.5))


def test_device_results_match_host_results(ctx):
    scenes, rng = _scenes(ctx, [80_000, 200_000], 10)
    views = [_view(rng) for _ in range(6)]
    with Server(ctx, memory_budget=1 << 30) as srv:
        host = [srv.wait(srv.submit(scenes[k % 2][1], make_view(v.model_view, v.projection, v.viewport, v.cull)))
                for k, v in enumerate(views)]
        tickets = [srv.submit(scenes[k % 2][1], make_view(v.model_view, v.projection, v.viewport, v.cull))
                   for k, v in enumerate(views)]
        for t, (order, keys) in zip(tickets, host):
            o_ptr, k_ptr, count = srv.result(t)
            assert count == order.size
            assert np.array_equal(ctx.download(o_ptr, count * 4), order)
            assert np.array_equal(ctx.download(k_ptr, count * 4), keys)
            srv.release(t)
    for _, sp, _ in scenes:
        sp.destroy()
