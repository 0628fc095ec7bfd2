"""Failures made on the host, each leaving the library usable: device
allocations refused through the injection hook, and requests withdrawn from
the serving loop while others complete. No GPU fault is caused."""
import numpy as np
import pytest

from oracle import oracle as O
from winding_b200 import Context, WsError, _lib, make_view, parse_splats, workloads as W
from winding_b200.server import Server

pytestmark = pytest.mark.gpu


def _scene(ctx, n, seed, kind="cluster"):
    rec = W.scene(kind, n, seed)
    return parse_splats(rec, ctx), O.parse_splat(rec.tobytes())


def _view(rng, cull=0.5):
    return W.View(W.random_pose(rng), W.perspective(W.FOV_Y, W.ASPECT, W.NEAR), W.VIEWPORT, cull)


def _ws(v):
    return make_view(v.model_view, v.projection, v.viewport, v.cull)


@pytest.fixture
def fresh():
    """A context whose device buffers have not grown yet."""
    c = Context(0)
    yield c
    _lib.load().ws_inject_alloc_failures(0)
    c.close()


def test_refused_allocation_fails_the_call_and_the_next_succeeds(fresh):
    rng = np.random.default_rng(21)
    sp, parsed = _scene(fresh, 200_000, 21)
    try:
        v = _view(rng)
        want_o, want_k = O.sort_view(parsed, v.model_view, v.projection, v.viewport, v.cull)
        assert fresh.lib.ws_inject_alloc_failures(3) == _lib.WS_OK
        for _ in range(3):
            with pytest.raises(WsError, match="out of device memory") as e:
                fresh.sort(sp, _ws(v))
            assert e.value.code == _lib.WS_ERR_NOMEM
        order, keys = fresh.sort(sp, _ws(v))
        assert np.array_equal(order, want_o) and np.array_equal(keys, want_k)
    finally:
        sp.destroy()


def test_refused_allocation_in_the_draw(fresh, ctx):
    import torch
    rng = np.random.default_rng(22)
    sp, _ = _scene(fresh, 50_000, 22)
    ref, _ = _scene(ctx, 50_000, 22)
    w, h = 160, 90
    try:
        v = W.View(W.random_pose(rng), W.perspective(W.FOV_Y, w / h, W.NEAR), (float(w), float(h)), 0.5)
        images = []
        for c, s in ((fresh, sp), (ctx, ref)):
            o = torch.empty(s.count, dtype=torch.int32, device="cuda")
            k = torch.empty_like(o)
            n = torch.zeros(1, dtype=torch.int32, device="cuda")
            c.sort_device(s, _ws(v), o.data_ptr(), k.data_ptr(), n.data_ptr())
            img = torch.zeros((h, w, 4), dtype=torch.float32, device="cuda")
            if c is fresh:
                c.sync()
                assert c.lib.ws_inject_alloc_failures(1) == _lib.WS_OK
                with pytest.raises(WsError, match="out of device memory"):
                    c.draw(s, _ws(v), o.data_ptr(), n.data_ptr(), img.data_ptr(), w, h)
            c.draw(s, _ws(v), o.data_ptr(), n.data_ptr(), img.data_ptr(), w, h)
            c.sync()
            images.append(img.cpu().numpy())
        assert np.array_equal(images[0].view(np.uint32), images[1].view(np.uint32))
        assert images[0][..., 3].any()
    finally:
        sp.destroy()
        ref.destroy()


def test_cancelled_requests_while_others_complete(ctx):
    rng = np.random.default_rng(23)
    scenes = [_scene(ctx, n, 230 + j, W.KINDS[j % 3]) for j, n in enumerate([120_000, 40_000, 300_000])]
    views = [_view(rng) for _ in range(8)]
    # A long collection window keeps every request queued until it fills.
    with Server(ctx, memory_budget=1 << 30, max_batch=64, collect_us=3_000_000) as srv:
        tickets = [srv.submit(scenes[k % 3][0], _ws(v)) for k, v in enumerate(views)]
        withdrawn = {1, 4, 6}
        for k in sorted(withdrawn):
            assert srv.cancel(tickets[k])
        with pytest.raises(WsError, match="WS_ERR_ARG"):
            srv.cancel(tickets[1])                      # already withdrawn: unknown
        kept = [k for k in range(len(views)) if k not in withdrawn]
        results = {k: srv.wait(tickets[k]) for k in kept}
        with pytest.raises(WsError, match="WS_ERR_ARG"):
            srv.wait(tickets[4], timeout_ms=0)
        # A request already dispatched cannot be withdrawn; collect it.
        t = srv.submit(scenes[0][0], _ws(views[0]))
        o_ptr, k_ptr, count = srv.result(t)
        assert not srv.cancel(t)
        assert count == results[0][0].size
        srv.release(t)
        st = srv.stats()
    assert st["cancelled"] == 3 and st["completed"] == len(kept) + 1 and st["failed"] == 0
    for k in kept:
        v = views[k]
        want_o, want_k = O.sort_view(scenes[k % 3][1], v.model_view, v.projection, v.viewport, v.cull)
        assert np.array_equal(results[k][0], want_o) and np.array_equal(results[k][1], want_k)
    for sp, _ in scenes:
        sp.destroy()


def test_cancelling_everything_queued_leaves_the_loop_serving(ctx):
    rng = np.random.default_rng(24)
    sp, parsed = _scene(ctx, 80_000, 24)
    try:
        with Server(ctx, memory_budget=1 << 28, max_batch=32, collect_us=3_000_000) as srv:
            tickets = [srv.submit(sp, _ws(_view(rng))) for _ in range(10)]
            assert all(srv.cancel(t) for t in tickets)
            v = _view(rng)
            order, keys = srv.wait(srv.submit(sp, _ws(v)))
            st = srv.stats()
        want_o, want_k = O.sort_view(parsed, v.model_view, v.projection, v.viewport, v.cull)
        assert np.array_equal(order, want_o) and np.array_equal(keys, want_k)
        assert st["cancelled"] == 10 and st["completed"] == 1
    finally:
        sp.destroy()
