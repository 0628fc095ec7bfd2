"""The splat draw (render/splats.js:252-312) into a headless RGBA f32 image.

CPU: the library's decodeSRGB and log tables against the oracle's (computed
independently, in long double), and the oracle's draw on hand-checked cases.
GPU: sort then ws_draw against the oracle's draw of the oracle's order, bit
for bit, over a background, with shaded colours, an empty order and the
refusals.
"""
import numpy as np
import pytest

from oracle import oracle as O
from winding_b200 import camera, workloads as W
from winding_b200.splats import draw_tables


def test_tables_match_the_oracle():
    srgb, reach = draw_tables()
    o_srgb, o_reach = O.draw_tables()
    assert np.array_equal(srgb.view(np.uint32), o_srgb.view(np.uint32))
    assert np.array_equal(reach.view(np.uint32), o_reach.view(np.uint32))
    assert srgb[0] == 0 and srgb[255] == 1.0
    assert reach[1] == 0 and np.isneginf(reach[0])


def _one_splat(alpha_byte=255, scale=0.05):
    rec = np.zeros(1, W.RECORD)
    rec["scale"] = scale
    rec["rgba"] = [255, 128, 0, alpha_byte]
    rec["rot"] = [255, 128, 128, 128]
    return rec


def test_oracle_draws_one_splat_at_the_centre():
    rec = _one_splat(scale=0.3)   # about 3 pixels across its sigma
    parsed = O.parse_splat(rec.tobytes())
    mv = camera.look_at((0, 0, 5), (0, 0, 0))
    proj = camera.perspective(np.pi / 3, 1.0, 0.1)
    img = O.draw(parsed, [0], mv, proj, 64, 64)
    a = img[..., 3]
    cy, cx = np.unravel_index(np.argmax(a), a.shape)
    assert (cy, cx) in [(31, 31), (31, 32), (32, 31), (32, 32)]
    assert 0.9 < a.max() <= 0.99
    assert np.allclose(img[..., 0], a * 1.0) and np.all(img[..., 2] == 0)   # red 255, blue 0: premultiplied
    assert np.all(a[0, :] == 0)                                               # a small splat: edges untouched
    faint = O.draw(O.parse_splat(_one_splat(alpha_byte=1, scale=0.3).tobytes()), [0], mv, proj, 64, 64)
    assert not faint.any()                                                    # reach <= 0: not drawn


def _cut_cases():
    """Clouds for the box cut's check: seeded scale spreads from specks to
    splats wider than the image, seen close up, at odd and large sizes."""
    for seed in range(14):
        if seed in (11, 13):   # the two slowest (billions of box pixels); the others cover their ranges
            continue
        rng = np.random.default_rng(100 + seed)
        n = 3000
        rec = W.records_from(rng.uniform(-10, 10, size=(n, 3)), rng)
        rec["scale"] = np.exp(rng.normal([-5.0, -3.0, -1.5, -0.5][seed % 4], 1.5, size=(n, 3))).astype(np.float32)
        w, h = [(64, 48), (333, 197), (1920, 1080), (4096, 2160)][(seed // 4) % 4]
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        mv = W.look_at(d * rng.uniform(6, 40), (0, 0, 0))
        yield rec.tobytes(), mv, camera.perspective(W.FOV_Y, w / h, W.NEAR), w, h


def test_box_cut_leaves_no_covered_pixel_out():
    """The draw keeps, of each splat's pinned pixel box, the pixels within
    the quad's half-extents (plus a margin); the oracle's coverage test,
    pixel by pixel, finds no covered pixel outside that cut on the bench's
    draw, the real capture and clouds of extreme scales and sizes."""
    import os
    cases = list(_cut_cases())
    job = W.clusters_1m(seed=1)
    cases.append((job.bytes(), job.view.model_view, job.view.projection, 1920, 1080))
    for name in ("cactus_posed_16384", "cactus_front_16384"):
        g = np.load(os.path.join(os.path.dirname(__file__), "golden", f"{name}.npz"))
        cases.append((g["records"].tobytes(), g["model_view"], g["projection"], 1920, 1080))
    covered = box = cut = 0
    for data, mv, pr, w, h in cases:
        parsed = O.parse_splat(data)
        order, _ = O.sort_view(parsed, mv, pr, (float(w), float(h)), 0.0, threads=4)
        missed, c, b, k = O.draw_cut_check(parsed, order, mv, pr, w, h)
        assert missed == 0
        covered, box, cut = covered + c, box + b, cut + k
    assert covered > 10**7 and cut < box


def _sorted(ctx, job, cull=0.5):
    import torch
    from winding_b200 import make_view, parse_splats
    sp = parse_splats(job.records, ctx)
    view = make_view(job.view.model_view, job.view.projection, job.view.viewport, cull)
    o = torch.empty(sp.count, dtype=torch.int32, device="cuda")
    k = torch.empty_like(o)
    c = torch.zeros(1, dtype=torch.int32, device="cuda")
    ctx.sort_device(sp, view, o.data_ptr(), k.data_ptr(), c.data_ptr())
    return sp, view, o, c


def _job(n, seed, w, h):
    job = W.clusters_1m(seed=seed, n=n)
    proj = camera.perspective(W.FOV_Y, w / h, W.NEAR)
    job.view = W.View(job.view.model_view, proj, (float(w), float(h)), 0.5)
    return job


@pytest.mark.gpu
@pytest.mark.parametrize("w,h", [(480, 270), (333, 197)])
def test_draw_matches_oracle(ctx, w, h):
    import torch
    job = _job(150_000, 5, w, h)
    sp, view, o, c = _sorted(ctx, job)
    try:
        rng = np.random.default_rng(1)
        bg = rng.uniform(0, 1, size=(h, w, 4)).astype(np.float32)
        img = torch.from_numpy(bg.copy()).cuda()
        ctx.draw(sp, view, o.data_ptr(), c.data_ptr(), img.data_ptr(), w, h)
        ctx.sync()
        got = img.cpu().numpy()
        order = o[: int(c.item())].cpu().numpy().view(np.uint32)
        want = O.draw(O.parse_splat(job.bytes()), order, job.view.model_view, job.view.projection, w, h,
                      background=bg)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
        assert (got != bg).mean() > 0.05
    finally:
        sp.destroy()


@pytest.mark.gpu
@pytest.mark.parametrize("crowd_min", [0, 1, 256])
def test_crowded_tile_kernel_matches_oracle(ctx, crowd_min):
    """Every tile through the crowded-tile kernel (1), none (0), and a split
    (256): the same image, bit for bit, as the oracle's."""
    import torch
    from winding_b200 import WsError
    w, h = 480, 270
    job = _job(150_000, 8, w, h)
    sp, view, o, c = _sorted(ctx, job)
    try:
        ctx.set_draw_crowded(crowd_min)
        rng = np.random.default_rng(2)
        bg = rng.uniform(0, 1, size=(h, w, 4)).astype(np.float32)
        img = torch.from_numpy(bg.copy()).cuda()
        ctx.draw(sp, view, o.data_ptr(), c.data_ptr(), img.data_ptr(), w, h)
        ctx.sync()
        order = o[: int(c.item())].cpu().numpy().view(np.uint32)
        want = O.draw(O.parse_splat(job.bytes()), order, job.view.model_view, job.view.projection, w, h,
                      background=bg)
        assert np.array_equal(img.cpu().numpy().view(np.uint32), want.view(np.uint32))
        with pytest.raises(WsError, match="power of two"):
            ctx.set_draw_crowded(1000)
    finally:
        ctx.set_draw_crowded(256)
        sp.destroy()


@pytest.mark.gpu
@pytest.mark.parametrize("crowd_min", [1, 256, 1024])
def test_draw_of_the_real_capture(ctx, crowd_min):
    """16,384 splats of the reference's real capture (the cactus fixture),
    sorted and drawn at 1920 x 1080, against the oracle's draw."""
    import os
    import torch
    from winding_b200 import make_view, parse_splats
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "cactus_posed_16384.npz"))
    w, h = (int(v) for v in g["viewport"])
    sp = parse_splats(g["records"].tobytes(), ctx)
    try:
        ctx.set_draw_crowded(crowd_min)
        view = make_view(g["model_view"], g["projection"], tuple(g["viewport"]), 0.5)
        o = torch.empty(sp.count, dtype=torch.int32, device="cuda")
        k = torch.empty_like(o)
        c = torch.zeros(1, dtype=torch.int32, device="cuda")
        ctx.sort_device(sp, view, o.data_ptr(), k.data_ptr(), c.data_ptr())
        img = torch.zeros((h, w, 4), dtype=torch.float32, device="cuda")
        ctx.draw(sp, view, o.data_ptr(), c.data_ptr(), img.data_ptr(), w, h)
        ctx.sync()
        order = o[: int(c.item())].cpu().numpy().view(np.uint32)
        assert np.array_equal(order, g["order_0p5"])
        want = O.draw(O.parse_splat(g["records"].tobytes()), order, g["model_view"], g["projection"], w, h)
        got = img.cpu().numpy()
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
        assert (got[..., 3] > 0).mean() > 0.01
    finally:
        ctx.set_draw_crowded(256)
        sp.destroy()


@pytest.mark.gpu
def test_bench_workload_draw_1m(ctx):
    """The bench's draw, whole: clusters-1M sorted and drawn at 1920 x 1080,
    bit for bit against the oracle's draw of the oracle's order."""
    import torch
    job = W.clusters_1m(seed=1)
    sp, view, o, c = _sorted(ctx, job)
    try:
        img = torch.zeros((1080, 1920, 4), dtype=torch.float32, device="cuda")
        ctx.draw(sp, view, o.data_ptr(), c.data_ptr(), img.data_ptr(), 1920, 1080)
        ctx.sync()
        order = o[: int(c.item())].cpu().numpy().view(np.uint32)
        want = O.draw(O.parse_splat(job.bytes()), order, job.view.model_view, job.view.projection, 1920, 1080)
        assert np.array_equal(img.cpu().numpy().view(np.uint32), want.view(np.uint32))
    finally:
        sp.destroy()


@pytest.mark.gpu
def test_draw_with_shaded_colours(ctx):
    import torch
    from winding_b200.splats import eye_in_cloud
    w, h = 320, 180
    job = _job(60_000, 6, w, h)
    from winding_b200 import make_view, parse_splats
    sp = parse_splats(job.records, ctx)
    try:
        sp.set_harmonics(2, W.harmonics_words(sp.count, 2))
        view = make_view(job.view.model_view, job.view.projection, job.view.viewport, 0.5)
        o = torch.empty(sp.count, dtype=torch.int32, device="cuda")
        k = torch.empty_like(o)
        c = torch.zeros(1, dtype=torch.int32, device="cuda")
        shaded = torch.zeros(sp.count, dtype=torch.int32, device="cuda")
        ctx.sort_batch_shaded([(sp, view, o.data_ptr(), k.data_ptr(), c.data_ptr())],
                              [(eye_in_cloud(job.view.model_view), shaded.data_ptr())])
        img = torch.zeros((h, w, 4), dtype=torch.float32, device="cuda")
        ctx.draw(sp, view, o.data_ptr(), c.data_ptr(), img.data_ptr(), w, h, shaded.data_ptr())
        ctx.sync()
        order = o[: int(c.item())].cpu().numpy().view(np.uint32)
        want = O.draw(O.parse_splat(job.bytes()), order, job.view.model_view, job.view.projection, w, h,
                      shaded=shaded.cpu().numpy().view(np.uint32))
        assert np.array_equal(img.cpu().numpy().view(np.uint32), want.view(np.uint32))
    finally:
        sp.destroy()


@pytest.mark.gpu
def test_draw_nothing_and_refusals(ctx):
    import torch
    from winding_b200 import WsError
    w, h = 128, 96
    job = _job(20_000, 7, w, h)
    sp, view, o, c = _sorted(ctx, job)
    try:
        img = torch.full((h, w, 4), 0.25, dtype=torch.float32, device="cuda")
        zero = torch.zeros(1, dtype=torch.int32, device="cuda")
        ctx.draw(sp, view, o.data_ptr(), zero.data_ptr(), img.data_ptr(), w, h)
        ctx.sync()
        assert torch.all(img == 0.25)
        with pytest.raises(WsError, match="viewport"):
            ctx.draw(sp, view, o.data_ptr(), c.data_ptr(), img.data_ptr(), w + 1, h)
        with pytest.raises(WsError, match="16-byte aligned"):
            ctx.draw(sp, view, o.data_ptr(), c.data_ptr(), img.data_ptr() + 4, w, h)
        with pytest.raises(WsError, match="1 to 4096"):
            ctx.draw(sp, view, o.data_ptr(), c.data_ptr(), img.data_ptr(), 0, h)
    finally:
        sp.destroy()
