"""The one-CTA sorts (ws_params.algorithm 1: two 8-bit passes in shared
memory; 2: one counting pass over all 65536 keys) against the oracle, bit
for bit: ragged sizes up to the largest job they take, the views that
exercise the general paths, batches and plans of small jobs, launches they
do not take (a job above 16384 splats), host outputs and the fused shade."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.test_parity_gpu import _adversarial_cloud, _device_jobs, _results, check_job, oracle_sort
from winding_b200 import _lib, make_view, parse_splats, workloads as W

pytestmark = pytest.mark.gpu

ALGOS = [_lib.ALGO_ONE_RADIX, _lib.ALGO_ONE_COUNT]


@pytest.fixture(params=ALGOS, ids=["one-radix", "one-count"])
def algo_ctx(ctx, request):
    old = ctx.params
    ctx.set_params(algorithm=request.param)
    try:
        yield ctx
    finally:
        ctx.set_params(tile=old.tile, ctas_per_sm=old.ctas_per_sm, segs_per_cta=old.segs_per_cta,
                       algorithm=old.algorithm)


@pytest.mark.parametrize("n", [1, 2, 31, 32, 33, 255, 257, 1000, 4097, 12289, 16383, 16384, 16385])
def test_ragged_sizes(algo_ctx, n):
    check_job(algo_ctx, W.uniform_100k(seed=300 + n, n=n))


@pytest.mark.parametrize("n", [5000, 16384])
def test_clusters_and_slab(algo_ctx, n):
    check_job(algo_ctx, W.clusters_1m(seed=31, n=n), culls=(0.0, 0.5, 2.0))
    check_job(algo_ctx, W.slab_6m(seed=32, n=n))   # many equal keys


@pytest.mark.parametrize("kind", ["persp-close", "ortho", "offcentre", "nonaffine"])
def test_general_views(algo_ctx, kind):
    from winding_b200.camera import look_at, perspective
    rec = _adversarial_cloud(12_000, 170 + len(kind), -2.0 if kind == "persp-close" else -3.5, 1.0)
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
    check_job(algo_ctx, W.Job(rec, W.View(mv, proj, (1280.0, 720.0), 0.5)), culls=(0.0, 0.5, 1.0, 3.0))


def test_behind_and_all_faint(algo_ctx):
    from winding_b200.camera import look_at, perspective
    job = W.uniform_100k(seed=19, n=3000)
    sp = parse_splats(job.records, algo_ctx)
    order, _ = algo_ctx.sort(sp, make_view(look_at((0, 0, 500), (0, 0, 1000)), perspective(0.8, 4 / 3, 0.1),
                                           (160, 120), 0.5))
    assert order.size == 0
    sp.destroy()
    job.records["rgba"][:, 3] = 1
    check_job(algo_ctx, job)


def test_batch_and_plan_of_small_jobs(algo_ctx):
    import torch
    rng = np.random.default_rng(17)
    jobs = []
    for j in range(12):
        n = int(rng.integers(1, _lib.ONE_CTA_MAX + 1)) if j else _lib.ONE_CTA_MAX
        rec = W.scene(W.KINDS[j % 3], n, 900 + j)
        jobs.append(W.Job(rec, W.View(W.random_pose(rng), W.perspective(W.FOV_Y, W.ASPECT, W.NEAR))))
    culls = [0.5 if j % 2 else 0.0 for j in range(len(jobs))]
    outs, specs = _device_jobs(algo_ctx, jobs, culls)
    stream = torch.cuda.current_stream().cuda_stream
    try:
        algo_ctx.sort_batch(specs, stream=stream)
        for (order, keys), job, cull in zip(_results(outs), jobs, culls):
            want_o, want_k = oracle_sort(O.parse_splat(job.bytes()), job.view, cull)
            assert np.array_equal(order, want_o) and np.array_equal(keys, want_k)
        plan = algo_ctx.plan(specs)
        views = []
        for job, cull in zip(jobs, culls):
            job.view.model_view = W.random_pose(rng)
            views.append(make_view(job.view.model_view, job.view.projection, job.view.viewport, cull))
        plan.set_views(views)
        plan.launch(stream)
        for (order, keys), job, cull in zip(_results(outs), jobs, culls):
            want_o, want_k = oracle_sort(O.parse_splat(job.bytes()), job.view, cull)
            assert np.array_equal(order, want_o) and np.array_equal(keys, want_k)
        plan.close()
    finally:
        for sp, *_ in outs:
            sp.destroy()


def test_a_large_job_sends_the_launch_to_the_three_phases(algo_ctx):
    """One job above the limit: the whole batch takes the three phases,
    with the same results."""
    import torch
    rng = np.random.default_rng(23)
    jobs = [W.Job(W.scene(W.KINDS[j], n, 950 + j), W.View(W.random_pose(rng), W.perspective(W.FOV_Y, W.ASPECT,
                                                                                             W.NEAR)))
            for j, n in enumerate((900, 40_000, 16_000))]
    outs, specs = _device_jobs(algo_ctx, jobs, [0.5] * 3)
    try:
        algo_ctx.sort_batch(specs, stream=torch.cuda.current_stream().cuda_stream)
        for (order, keys), job in zip(_results(outs), jobs):
            want_o, want_k = oracle_sort(O.parse_splat(job.bytes()), job.view, 0.5)
            assert np.array_equal(order, want_o) and np.array_equal(keys, want_k)
    finally:
        for sp, *_ in outs:
            sp.destroy()


def test_host_outputs_and_no_keys(algo_ctx):
    import ctypes

    import torch
    job = W.clusters_1m(seed=61, n=9000)
    sp = parse_splats(job.records, algo_ctx)
    view = make_view(job.view.model_view, job.view.projection, job.view.viewport, 0.5)
    want_o, want_k = oracle_sort(O.parse_splat(job.bytes()), job.view, 0.5)
    order = torch.full((sp.count,), -1, dtype=torch.int32).pin_memory()
    cnt = ctypes.c_uint32()
    for buf in (order, torch.full((sp.count,), -1, dtype=torch.int32)):   # pinned, then pageable
        algo_ctx.check(algo_ctx.lib.ws_sort(algo_ctx.handle, sp.handle, ctypes.byref(view), buf.data_ptr(), None,
                                            ctypes.byref(cnt), _lib.WS_HOST_OUTPUT, None))
        assert cnt.value == want_o.size
        assert np.array_equal(buf[:cnt.value].numpy().view(np.uint32), want_o)
    sp.destroy()


def test_fused_shade_matches_the_three_phases(algo_ctx):
    import torch
    from winding_b200.splats import eye_in_cloud
    job = W.clusters_1m(seed=71, n=12_000)
    sp = parse_splats(job.records, algo_ctx)
    sp.set_harmonics(3, W.harmonics_words(sp.count, 3))
    view = make_view(job.view.model_view, job.view.projection, job.view.viewport, 0.5)
    eye = eye_in_cloud(job.view.model_view)
    res = []
    for algorithm in (_lib.ALGO_PHASES, algo_ctx.params.algorithm):
        algo_ctx.set_params(algorithm=algorithm)
        o = torch.empty(sp.count, dtype=torch.int32, device="cuda")
        k = torch.empty_like(o)
        c = torch.zeros(1, dtype=torch.int32, device="cuda")
        shaded = torch.zeros_like(o)
        algo_ctx.sort_batch_shaded([(sp, view, o.data_ptr(), k.data_ptr(), c.data_ptr())],
                                   [(eye, shaded.data_ptr())])
        algo_ctx.sync()
        s = int(c.item())
        live = o[:s].long()
        res.append((o[:s].cpu().numpy(), k[:s].cpu().numpy(), shaded[live].cpu().numpy()))
    assert all(np.array_equal(a, b) for a, b in zip(*res))
    sp.destroy()


def test_unknown_algorithm_is_refused(ctx):
    from winding_b200 import WsError
    with pytest.raises(WsError, match="algorithm"):
        ctx.set_params(algorithm=3)
    assert ctx.params.algorithm == _lib.ALGO_PHASES
