"""GPU parity: libwsort.so against the CPU oracle, bit for bit.

Every comparison is exact (np.array_equal on u32 / the f32 bit patterns):
the only floating-point steps are pinned to separately rounded IEEE ops on
both sides, and everything after them is integer work.
"""
import glob
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests import kats
from winding_b200 import WsError, make_view, parse_splats, workloads as W
from winding_b200 import _lib

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def oracle_sort(parsed, view_src, cull):
    return O.sort_view(parsed, view_src.model_view, view_src.projection, view_src.viewport, cull)


def check_job(ctx, job, culls=(0.0, 0.5)):
    splats = parse_splats(job.records, ctx)
    parsed = O.parse_splat(job.bytes())
    try:
        for cull in culls:
            view = make_view(job.view.model_view, job.view.projection, job.view.viewport, cull)
            order, keys = ctx.sort(splats, view)
            want_o, want_k = oracle_sort(parsed, job.view, cull)
            assert order.size == want_o.size, (cull, order.size, want_o.size)
            assert np.array_equal(order, want_o), cull
            assert np.array_equal(keys, want_k), cull
    finally:
        splats.destroy()


def test_decode_matches_the_oracle(ctx):
    job = W.clusters_1m(seed=31, n=50_000)
    splats = parse_splats(job.records, ctx)
    parsed = O.parse_splat(job.bytes())
    c, v = splats.download()
    assert np.array_equal(c.view(np.uint32), parsed.centers.view(np.uint32))
    assert np.array_equal(v.view(np.uint32), parsed.covariances.view(np.uint32))
    assert splats.min == list(parsed.min) and splats.max == list(parsed.max)
    splats.destroy()


def test_decode_known_answers(ctx):
    s = parse_splats(kats.UNTURNED, ctx)
    c, v = s.download()
    assert list(c[0, :3]) == [1, 2, 3]
    assert list(c.view(np.uint8).reshape(-1, 16)[0, 12:]) == [10, 20, 30, 200]
    assert np.allclose(v[0], kats.UNTURNED_COV, atol=1e-4)
    q = parse_splats(kats.QUARTER, ctx)
    _, v = q.download()
    assert abs(v[0, 0] - 4) <= 1e-2 and abs(v[0, 3] - 0.25) <= 1e-2 and abs(v[0, 1]) <= 1e-2


@pytest.mark.parametrize("data,message", kats.REFUSED)
def test_refusals_by_message(ctx, data, message):
    with pytest.raises(WsError, match=message):
        parse_splats(data, ctx)


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "*.npz"))))
def test_golden_fixtures(ctx, path):
    g = np.load(path)
    splats = parse_splats(g["records"], ctx)
    for tag, cull in (("0p0", 0.0), ("0p5", 0.5)):
        order, keys = ctx.sort(splats, make_view(g["model_view"], g["projection"], g["viewport"], cull))
        assert np.array_equal(order, g[f"order_{tag}"]), (path, cull)
        assert np.array_equal(keys, g[f"keys_{tag}"]), (path, cull)
    splats.destroy()


@pytest.mark.parametrize("n", [1, 2, 31, 32, 33, 255, 256, 257, 2047, 2048, 2049, 4095, 4096, 4097, 12289])
def test_ragged_sizes(ctx, n):
    check_job(ctx, W.uniform_100k(seed=100 + n, n=n))


def test_uniform_100k(ctx):
    check_job(ctx, W.uniform_100k(seed=0), culls=(0.0, 0.5, 2.0))


def test_clusters_300k(ctx):
    check_job(ctx, W.clusters_1m(seed=1, n=300_000))


def test_slab_heavy_collisions(ctx):
    check_job(ctx, W.slab_6m(seed=2, n=400_000))


@pytest.mark.parametrize("red_first", [True, False])
def test_two_splats_back_to_front(ctx, red_first):
    s = parse_splats(kats.two_splats(red_first), ctx)
    red, blue = (0, 1) if red_first else (1, 0)
    mv, proj, vp = kats.gpu_test_camera(5.0)
    order, keys = ctx.sort(s, make_view(mv, proj, vp, 0.5))
    assert list(order) == [blue, red] and list(keys) == [0, 65535]
    mv, proj, vp = kats.gpu_test_camera(-5.0)
    order, _ = ctx.sort(s, make_view(mv, proj, vp, 0.5))
    assert list(order) == [red, blue]
    s.destroy()


def test_single_splat_and_speck(ctx):
    mv, proj, vp = kats.gpu_test_camera(5.0)
    one = parse_splats(kats.two_splats(True)[:32], ctx)
    order, keys = ctx.sort(one, make_view(mv, proj, vp, 0.5))
    assert list(order) == [0] and list(keys) == [65535]
    speck = parse_splats(kats.speck_file(), ctx)
    assert list(ctx.sort(speck, make_view(mv, proj, vp, 0.5))[0]) == [1]
    assert sorted(ctx.sort(speck, make_view(mv, proj, vp, 0.0))[0]) == [0, 1]


def test_behind_the_camera_and_all_culled(ctx):
    from winding_b200.camera import look_at, perspective
    s = parse_splats(kats.two_splats(True), ctx)
    order, _ = ctx.sort(s, make_view(look_at((0, 0, 5), (0, 0, 10)), perspective(0.8, 4 / 3, 0.1), (160, 120), 0.5))
    assert order.size == 0
    # In front, but every splat too faint.
    job = W.uniform_100k(seed=9, n=5000)
    job.records["rgba"][:, 3] = 1
    check_job(ctx, job)


def test_cull_errors_and_unloaded(ctx):
    s = parse_splats(kats.two_splats(True), ctx)
    mv, proj, vp = kats.gpu_test_camera(5.0)
    with pytest.raises(WsError, match="splatCull must be 0 or more, got -1"):
        ctx.sort(s, make_view(mv, proj, vp, -1.0))
    s.destroy()
    with pytest.raises(WsError, match="unloaded"):
        ctx.sort(s, make_view(mv, proj, vp, 0.5))
    rc = ctx.lib.ws_sort(ctx.handle, s.handle, None, None, None, None, 0, None)
    assert rc == _lib.WS_ERR_UNLOADED


def _device_jobs(ctx, jobs, culls):
    import torch
    outs = []
    specs = []
    for job, cull in zip(jobs, culls):
        sp = parse_splats(job.records, ctx)
        n = max(sp.count, 1)
        o = torch.empty(n, dtype=torch.int32, device="cuda")
        k = torch.empty(n, dtype=torch.int32, device="cuda")
        c = torch.zeros(1, dtype=torch.int32, device="cuda")
        outs.append((sp, o, k, c))
        specs.append((sp, make_view(job.view.model_view, job.view.projection, job.view.viewport, cull),
                       o.data_ptr(), k.data_ptr(), c.data_ptr()))
    return outs, specs


def _results(outs):
    import torch
    torch.cuda.synchronize()
    res = []
    for sp, o, k, c in outs:
        s = int(c.item())
        res.append((o[:s].cpu().numpy().view(np.uint32), k[:s].cpu().numpy().view(np.uint32)))
    return res


def test_batch_equals_each_job_alone(ctx):
    import torch
    rng = np.random.default_rng(7)
    jobs = []
    for j in range(9):
        n = int(np.exp(rng.uniform(np.log(3_000), np.log(200_000))))
        rec = W.scene(W.KINDS[j % 3], n, 700 + j)
        jobs.append(W.Job(rec, W.View(W.random_pose(rng), W.perspective(W.FOV_Y, W.ASPECT, W.NEAR))))
    culls = [0.5 if j % 2 else 0.0 for j in range(len(jobs))]
    outs, specs = _device_jobs(ctx, jobs, culls)
    ctx.sort_batch(specs, stream=torch.cuda.current_stream().cuda_stream)
    got = _results(outs)
    ctx.sync()
    for (order, keys), job, cull in zip(got, jobs, culls):
        want_o, want_k = oracle_sort(O.parse_splat(job.bytes()), job.view, cull)
        assert np.array_equal(order, want_o) and np.array_equal(keys, want_k)
    # the graph-captured plan, twice, with new views the second time
    plan = ctx.plan(specs)
    plan.launch(torch.cuda.current_stream().cuda_stream)
    got2 = _results(outs)
    assert all(np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) for a, b in zip(got, got2))
    views = []
    for job, cull in zip(jobs, culls):
        job.view.model_view = W.random_pose(rng)
        views.append(make_view(job.view.model_view, job.view.projection, job.view.viewport, cull))
    plan.set_views(views)
    plan.launch(torch.cuda.current_stream().cuda_stream)
    got3 = _results(outs)
    for (order, keys), job, cull in zip(got3, jobs, culls):
        want_o, want_k = oracle_sort(O.parse_splat(job.bytes()), job.view, cull)
        assert np.array_equal(order, want_o) and np.array_equal(keys, want_k)
    plan.close()
    for sp, *_ in outs:
        sp.destroy()


# The bench's own workloads, whole, against the oracle: the configurations
# the throughput figures are measured on are the ones shown exact.

def test_bench_workload_clusters_1m(ctx):
    check_job(ctx, W.clusters_1m(seed=1))


def test_bench_workload_slab_6m(ctx):
    check_job(ctx, W.slab_6m(seed=2), culls=(0.5,))


def test_bench_workload_mixed_64_batched(ctx):
    import torch
    jobs = W.mixed_64(seed=3, cull=0.5)
    outs, specs = _device_jobs(ctx, jobs, [j.view.cull for j in jobs])
    try:
        ctx.sort_batch(specs, stream=torch.cuda.current_stream().cuda_stream)
        for (order, keys), job in zip(_results(outs), jobs):
            want_o, want_k = oracle_sort(O.parse_splat(job.bytes()), job.view, job.view.cull)
            assert np.array_equal(order, want_o) and np.array_equal(keys, want_k)
    finally:
        for sp, *_ in outs:
            sp.destroy()


# (least splats a segment covers, CTAs per SM, segments per CTA): one segment
# per job up to hundreds in many look-back groups, both kernel variants.
@pytest.mark.parametrize("tile,ctas,segs", [(2048, 1, 1), (2048, 2, 1), (8192, 1, 2), (1 << 20, 1, 1), (256, 1, 4),
                                            (256, 2, 4), (512, 2, 16), (1024, 1, 64)])
def test_kernel_variants_do_not_change_the_result(ctx, tile, ctas, segs):
    old = ctx.params
    try:
        ctx.set_params(tile=tile, ctas_per_sm=ctas, segs_per_cta=segs)
        check_job(ctx, W.clusters_1m(seed=41, n=120_001))
    finally:
        ctx.set_params(tile=old.tile, ctas_per_sm=old.ctas_per_sm, segs_per_cta=old.segs_per_cta)


def test_missing_kernel_variant_is_refused(ctx):
    old = ctx.params
    for tile, ctas, segs in [(777, 1, 1), (0, 1, 1), (128, 1, 1), (2048, 3, 1), (2048, 4, 1), (2048, 1, 65)]:
        with pytest.raises(WsError, match="tile|ctas_per_sm|segs_per_cta"):
            ctx.set_params(tile=tile, ctas_per_sm=ctas, segs_per_cta=segs)
    p = ctx.params
    assert (p.tile, p.ctas_per_sm, p.segs_per_cta) == (old.tile, old.ctas_per_sm, old.segs_per_cta)


def test_full_size_slab_properties(ctx):
    """6M splats: the oracle's result at full size, checked exactly, plus
    size-independent properties of the permutation."""
    job = W.slab_6m(seed=2)
    splats = parse_splats(job.records, ctx)
    parsed = O.parse_splat(job.bytes())
    view = make_view(job.view.model_view, job.view.projection, job.view.viewport, 0.5)
    order, keys = ctx.sort(splats, view)
    assert np.all(np.diff(keys.astype(np.int64)) >= 0)
    same = keys[1:] == keys[:-1]
    assert np.all(order[1:][same] > order[:-1][same])          # stable: index order within a key
    assert np.unique(order).size == order.size
    want_o, want_k = O.sort_view(parsed, job.view.model_view, job.view.projection, job.view.viewport, 0.5,
                                 threads=os.cpu_count() or 1)
    assert np.array_equal(order, want_o) and np.array_equal(keys, want_k)
    splats.destroy()


def _adversarial_cloud(n, seed, scale_mu, near_dist):
    rng = np.random.default_rng(seed)
    pos = rng.normal(size=(n, 3)) * np.array([2.0, 2.0, 2.0])
    rec = W.records_from(pos, rng)
    # wide spread of sizes: specks, thin needles and large blobs
    rec["scale"] = np.exp(rng.normal(scale_mu, 2.0, size=(n, 3))).astype(np.float32)
    flat = rng.random(n) < 0.2
    rec["scale"][flat, rng.integers(0, 3)] = 0.0          # rank-deficient covariances
    rec["rgba"][:, 3] = rng.integers(60, 80, size=n)      # alpha bytes around the shortcut's threshold
    return rec


@pytest.mark.parametrize("kind", ["persp-close", "persp-far", "ortho", "offcentre", "nonaffine"])
def test_views_that_exercise_the_general_paths(ctx, kind):
    from winding_b200.camera import look_at, perspective
    rng = np.random.default_rng({"persp-close": 1, "persp-far": 2, "ortho": 3, "offcentre": 4, "nonaffine": 5}[kind])
    rec = _adversarial_cloud(60_000, 70 + len(kind), -2.0 if kind == "persp-close" else -3.5, 1.0)
    dist = 6.0 if kind == "persp-close" else 40.0
    mv = look_at((dist * 0.3, dist * 0.2, dist), (0, 0, 0))
    proj = perspective(1.0, 16 / 9, 0.1)
    if kind == "ortho":
        proj = np.zeros(16, np.float32)
        proj[0], proj[5], proj[10], proj[14], proj[15] = 0.2, 0.35, -0.01, 0.5, 1.0
    elif kind == "offcentre":
        proj = proj.copy()
        proj[8], proj[9] = np.float32(0.15), np.float32(-0.1)
    elif kind == "nonaffine":
        mv = mv.copy()
        mv[3], mv[15] = np.float32(1e-3), np.float32(1.0001)
    job = W.Job(rec, W.View(mv, proj, (1280.0, 720.0), 0.5))
    check_job(ctx, job, culls=(0.0, 0.5, 1.0, 3.0))


def test_cull_threshold_sweep(ctx):
    """Culls around the footprint shortcut's bound; the same splats every time."""
    rec = _adversarial_cloud(40_000, 91, -4.0, 30.0)
    job = W.Job(rec, W.View(W.look_at((0, 0, 30), (0, 0, 0)), W.perspective(W.FOV_Y, W.ASPECT, W.NEAR)))
    check_job(ctx, job, culls=(0.3, 0.45, 0.4999, 0.5, 0.5001, 0.55, 0.7))


def test_tuning_table_changes_no_result(ctx):
    from winding_b200 import autotune
    job = W.clusters_1m(seed=81, n=150_000)
    splats = parse_splats(job.records, ctx)
    view = make_view(job.view.model_view, job.view.projection, job.view.viewport, 0.5)
    want = ctx.sort(splats, view)
    table = autotune.tune(ctx, [[(splats, view)]], reps=2)
    assert autotune.bucket(splats.count) in table
    got = ctx.sort(splats, view)
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
    bad = (_lib.WsParams * 1)()
    bad[0].tile = 777
    assert ctx.lib.ws_set_tuning(ctx.handle, bad, 1) == _lib.WS_ERR_ARG
    autotune.install(ctx, {})
    splats.destroy()


def test_a_wait_that_runs_out_is_reported_and_the_context_recovers(ctx):
    """Failure detection without a fault: a queued phase whose dependency
    never completes; its bounded wait gives up, the launch reports
    WS_ERR_TIMEOUT, and the next sort on the same context is exact."""
    from winding_b200 import _lib
    rc = ctx.lib.ws_selftest_wait(ctx.handle, 2000)
    assert rc == _lib.WS_ERR_TIMEOUT
    assert "device-side wait gave up" in ctx.lib.ws_last_error(ctx.handle).decode()
    check_job(ctx, W.uniform_100k(seed=77, n=50_000))


@pytest.mark.parametrize("pinned", [True, False])
def test_batch_with_host_outputs(ctx, pinned):
    """ws_sort_batch_host: every job's count, order and keys in host memory
    equal ws_sort_batch's device results (one copy kernel into pinned
    buffers, or counts then orders into pageable ones), twice in a row."""
    import ctypes

    import torch
    base = W.clusters_1m(seed=60, n=250_000)
    parts = [base.records[:70_001], base.records[:1], base.records[:0], base.records]
    clouds = [parse_splats(r, ctx) if len(r) else None for r in parts]
    try:
        live = [c for c in clouds if c is not None]
        specs, dev, host = [], [], []
        for sp in live:
            view = make_view(base.view.model_view, base.view.projection, base.view.viewport, 0.5)
            n = max(sp.count, 1)
            o = torch.empty(n, dtype=torch.int32, device="cuda")
            k = torch.empty(n, dtype=torch.int32, device="cuda")
            c = torch.zeros(1, dtype=torch.int32, device="cuda")
            dev.append((o, k, c))
            ho, hk, hc = (torch.full((n,), -1, dtype=torch.int32), torch.full((n,), -1, dtype=torch.int32),
                          torch.zeros(1, dtype=torch.int32))
            if pinned:
                ho, hk, hc = ho.pin_memory(), hk.pin_memory(), hc.pin_memory()
            host.append((ho, hk, hc))
            specs.append((sp, view))
        ctx.sort_batch([(sp, v, o.data_ptr(), k.data_ptr(), c.data_ptr()) for (sp, v), (o, k, c) in zip(specs, dev)])
        ctx.sync()
        for _ in range(2):
            ctx.copy_stats(reset=True)
            ctx.sort_batch_host([(sp, v, ho.data_ptr(), hk.data_ptr(), hc.data_ptr())
                                 for (sp, v), (ho, hk, hc) in zip(specs, host)])
            # the error words, then per job its count and its survivors' order and keys
            h2d, d2h = ctx.copy_stats()
            assert d2h == 8 + sum(4 + 8 * int(c.item()) for _, _, c in dev)
            assert h2d > 0
            for (o, k, c), (ho, hk, hc) in zip(dev, host):
                s = int(c.item())
                assert int(hc[0]) == s
                assert np.array_equal(ho[:s].numpy(), o[:s].cpu().numpy())
                assert np.array_equal(hk[:s].numpy(), k[:s].cpu().numpy())
    finally:
        for sp in clouds:
            if sp is not None:
                sp.destroy()


def test_host_output_into_pinned_buffers(ctx):
    """ws_sort with pinned host outputs takes the direct path (the survivors
    written into the host buffers by a kernel, one synchronisation); the
    result is the pageable path's, with and without keys, twice in a row."""
    import ctypes

    import torch

    from winding_b200 import _lib
    job = W.clusters_1m(seed=91, n=200_000)
    splats = parse_splats(job.records, ctx)
    view = make_view(job.view.model_view, job.view.projection, job.view.viewport, 0.5)
    try:
        want_o, want_k = ctx.sort(splats, view)
        order = torch.full((splats.count,), -1, dtype=torch.int32).pin_memory()
        keys = torch.full((splats.count,), -1, dtype=torch.int32).pin_memory()
        cnt = ctypes.c_uint32()
        for with_keys in (True, False, True):
            ctx.check(ctx.lib.ws_sort(ctx.handle, splats.handle, ctypes.byref(view), order.data_ptr(),
                                      keys.data_ptr() if with_keys else None, ctypes.byref(cnt),
                                      _lib.WS_HOST_OUTPUT, None))
            s = cnt.value
            assert s == len(want_o)
            assert np.array_equal(order[:s].numpy().view(np.uint32), want_o)
            if with_keys:
                assert np.array_equal(keys[:s].numpy().view(np.uint32), want_k)
    finally:
        splats.destroy()


def test_two_contexts_in_flight_at_once():
    """Two contexts sorting batches from two host threads at the same time
    (their kernels overlap on the device, as the pipelined bench runs them):
    every result is the oracle's."""
    import threading

    import torch

    from winding_b200 import Context
    rng = np.random.default_rng(29)
    jobs = [W.Job(W.scene(W.KINDS[j % 3], int(rng.integers(20_000, 300_000)), 970 + j),
                  W.View(W.random_pose(rng), W.perspective(W.FOV_Y, W.ASPECT, W.NEAR), cull=0.5))
            for j in range(8)]
    want = [oracle_sort(O.parse_splat(j.bytes()), j.view, 0.5) for j in jobs]
    ctxs = [Context(0), Context(0)]
    errors = []

    def run(c, k):
        try:
            clouds = [parse_splats(j.records, c) for j in jobs]
            host = [(torch.full((sp.count,), -1, dtype=torch.int32).pin_memory(),
                     torch.zeros(1, dtype=torch.int32).pin_memory()) for sp in clouds]
            specs = [(sp, make_view(j.view.model_view, j.view.projection, j.view.viewport, 0.5), ho.data_ptr(),
                      None, hc.data_ptr()) for sp, j, (ho, hc) in zip(clouds, jobs, host)]
            stream = torch.cuda.Stream()
            for _ in range(3):
                c.sort_batch_host(specs, stream.cuda_stream)
                for (ho, hc), (wo, _) in zip(host, want):
                    s = int(hc[0])
                    if s != wo.size or not np.array_equal(ho[:s].numpy().view(np.uint32), wo):
                        errors.append(k)
            for sp in clouds:
                sp.destroy()
        except Exception as exc:   # reported below, from the main thread
            errors.append(repr(exc))

    threads = [threading.Thread(target=run, args=(c, k)) for k, c in enumerate(ctxs)]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    for c in ctxs:
        c.close()
    assert not errors, errors
