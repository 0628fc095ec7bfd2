"""The shade pass (render/splats.js:315-382), fused into the sort's launch.

CPU: the oracle's shade against an independent numpy float32 restatement of
harmonics() (every op rounded to f32, left to right), and the identity that
all-zero harmonics leave a colour word as it is.
GPU: ws_sort_batch_shaded against the oracle for degrees 1, 2 and 3, only the
survivors' words written, the order and keys identical to the plain sort's;
a lone job shaded between plain sorts of the same size.
"""
import numpy as np
import pytest

from oracle import oracle as O
from winding_b200 import WsError, make_view, parse_splats, workloads as W
from winding_b200.splats import SH_WORDS, eye_in_cloud

COEFS = (0, 3, 8, 15)


def _sh_words(n, degree, rng, scale=0.4):
    """Random harmonics packed as the reference packs them."""
    per = SH_WORDS[degree]
    halves = np.zeros(n * per * 2 + 2, np.uint16)
    vals = (rng.uniform(-scale, scale, size=(n, COEFS[degree] * 3))).astype(np.float16)
    halves[: n * per * 2].reshape(n, per * 2)[:, : COEFS[degree] * 3] = vals.view(np.uint16)
    return halves.view(np.uint32)[: n * per + 1].copy()


def _np_shade(center, sh, degree, i, eye):
    f = np.float32
    per = SH_WORDS[degree]
    halves = sh.view(np.uint16)

    def coef(k):
        h = i * per * 2 + k * 3
        return halves[h:h + 3].view(np.float16).astype(np.float32)

    v = (center[:3] - eye).astype(np.float32)
    ln = np.sqrt(f(f(v[0] * v[0]) + f(v[1] * v[1])) + f(v[2] * v[2]))
    x, y, z = f(v[0] / ln), f(v[1] / ln), f(v[2] / ln)
    c = f(0.4886025119029199) * ((f(-y) * coef(0) + z * coef(1)) - x * coef(2))
    if degree >= 2:
        xx, yy, zz = f(x * x), f(y * y), f(z * z)
        K2, K3, K4 = f(1.0925484305920792), f(0.31539156525252005), f(0.5462742152960396)
        e = f(f(K2 * x) * y) * coef(3) - f(f(K2 * y) * z) * coef(4)
        e = e + f(K3 * f(f(f(2) * zz - xx) - yy)) * coef(5)
        e = e - f(f(K2 * x) * z) * coef(6)
        e = e + f(K4 * f(xx - yy)) * coef(7)
        c = c + e
        if degree >= 3:
            q = f(f(f(4) * zz - xx) - yy)
            a = f(f(f(-0.5900435899266435) * y) * f(f(3) * xx - yy))
            b = f(f(f(f(2.890611442640554) * x) * y) * z)
            cc = f(f(f(0.4570457994644658) * y) * q)
            d = f(f(f(0.3731763325901154) * z) * f(f(f(2) * zz - f(f(3) * xx)) - f(f(3) * yy)))
            ee = f(f(f(0.4570457994644658) * x) * q)
            ff = f(f(f(1.445305721320277) * z) * f(xx - yy))
            g = f(f(f(0.5900435899266435) * x) * f(xx - f(f(3) * yy)))
            h = a * coef(8) + b * coef(9)
            h = h - cc * coef(10)
            h = h + d * coef(11)
            h = h - ee * coef(12)
            h = h + ff * coef(13)
            h = h - g * coef(14)
            c = c + h
    word = int(center[3:4].view(np.uint32)[0])
    base = np.array([(word >> s) & 255 for s in (0, 8, 16, 24)], np.float32) / f(255)
    seen = np.clip(np.nan_to_num(base[:3] + c, nan=0.0), 0, 1).astype(np.float32)
    out = [int(np.floor(f(0.5) + f(255) * s)) for s in seen] + [int(np.floor(f(0.5) + f(255) * base[3]))]
    return out[0] | out[1] << 8 | out[2] << 16 | out[3] << 24


@pytest.mark.parametrize("degree", [1, 2, 3])
def test_oracle_shade_matches_numpy_restatement(degree):
    rng = np.random.default_rng(degree)
    rec = W.uniform(200, seed=degree)
    parsed = O.parse_splat(rec.tobytes())
    sh = _sh_words(parsed.count, degree, rng)
    eye = np.array([3.5, -20.0, 41.25], np.float32)
    got = O.shade(parsed.centers, sh, degree, range(parsed.count), eye)
    for i in range(parsed.count):
        assert got[i] == _np_shade(parsed.centers[i], sh, degree, i, eye), i


def test_zero_harmonics_keep_the_colour():
    rec = W.uniform(500, seed=9)
    parsed = O.parse_splat(rec.tobytes())
    words = parsed.centers.view(np.uint32)[:, 3]
    for degree in (1, 2, 3):
        sh = np.zeros(parsed.count * SH_WORDS[degree] + 1, np.uint32)
        got = O.shade(parsed.centers, sh, degree, range(parsed.count), np.zeros(3, np.float32))
        assert np.array_equal(got, words)


@pytest.mark.gpu
@pytest.mark.parametrize("degree", [1, 2, 3])
def test_sort_batch_shaded_matches_oracle(ctx, degree):
    import torch
    rng = np.random.default_rng(20 + degree)
    jobs = [W.clusters_1m(seed=50 + degree, n=150_000), W.uniform_100k(seed=60 + degree, n=30_000)]
    clouds, outs, specs, shades, want = [], [], [], [], []
    try:
        for job in jobs:
            sp = parse_splats(job.records, ctx)
            parsed = O.parse_splat(job.bytes())
            sh = _sh_words(sp.count, degree, rng)
            sp.set_harmonics(degree, sh)
            view = make_view(job.view.model_view, job.view.projection, job.view.viewport, 0.5)
            eye = eye_in_cloud(job.view.model_view)
            o = torch.empty(sp.count, dtype=torch.int32, device="cuda")
            k = torch.empty(sp.count, dtype=torch.int32, device="cuda")
            c = torch.zeros(1, dtype=torch.int32, device="cuda")
            shaded = torch.full((sp.count,), 0x5A5A5A5A, dtype=torch.int32, device="cuda")
            clouds.append(sp)
            outs.append((o, k, c, shaded))
            specs.append((sp, view, o.data_ptr(), k.data_ptr(), c.data_ptr()))
            shades.append((eye, shaded.data_ptr()))
            want.append((parsed, sh, eye, view))
        ctx.sort_batch_shaded(specs, shades)
        ctx.sync()
        for sp, (o, k, c, shaded), (parsed, sh, eye, view) in zip(clouds, outs, want):
            s = int(c.item())
            order = o[:s].cpu().numpy().view(np.uint32)
            keys = k[:s].cpu().numpy().view(np.uint32)
            plain_o, plain_k = ctx.sort(sp, view)
            assert np.array_equal(order, plain_o) and np.array_equal(keys, plain_k)
            got = shaded.cpu().numpy().view(np.uint32)
            expect = O.shade(parsed.centers, sh, degree, order, eye)
            assert np.array_equal(got[order], expect)
            untouched = np.ones(sp.count, bool)
            untouched[order] = False
            assert np.all(got[untouched] == 0x5A5A5A5A)
    finally:
        for sp in clouds:
            sp.destroy()


@pytest.mark.gpu
def test_bench_workload_shade_1m(ctx):
    """The bench's shade measurement, whole: clusters-1M with degree-3
    harmonics, sorted and shaded in one launch, every survivor's word
    against the oracle."""
    import torch
    rng = np.random.default_rng(41)
    job = W.clusters_1m(seed=1)
    sp = parse_splats(job.records, ctx)
    try:
        parsed = O.parse_splat(job.bytes())
        sh = _sh_words(sp.count, 3, rng)
        sp.set_harmonics(3, sh)
        view = make_view(job.view.model_view, job.view.projection, job.view.viewport, 0.5)
        eye = eye_in_cloud(job.view.model_view)
        o = torch.empty(sp.count, dtype=torch.int32, device="cuda")
        k = torch.empty_like(o)
        c = torch.zeros(1, dtype=torch.int32, device="cuda")
        shaded = torch.zeros(sp.count, dtype=torch.int32, device="cuda")
        ctx.sort_batch_shaded([(sp, view, o.data_ptr(), k.data_ptr(), c.data_ptr())], [(eye, shaded.data_ptr())])
        ctx.sync()
        order = o[:int(c.item())].cpu().numpy().view(np.uint32)
        got = shaded.cpu().numpy().view(np.uint32)
        assert np.array_equal(got[order], O.shade(parsed.centers, sh, 3, order, eye))
    finally:
        sp.destroy()


@pytest.mark.gpu
def test_lone_job_shaded_between_plain_sorts(ctx):
    """One job alone in its launch, sorted plain, then shaded, then plain
    again at the same size: each launch does its own work (the shade pass
    runs exactly when asked for), and the shaded words match the oracle."""
    import torch
    rng = np.random.default_rng(31)
    job = W.clusters_1m(seed=71, n=120_000)
    sp = parse_splats(job.records, ctx)
    try:
        parsed = O.parse_splat(job.bytes())
        sh = _sh_words(sp.count, 3, rng)
        sp.set_harmonics(3, sh)
        view = make_view(job.view.model_view, job.view.projection, job.view.viewport, 0.5)
        eye = eye_in_cloud(job.view.model_view)
        o = torch.empty(sp.count, dtype=torch.int32, device="cuda")
        k = torch.empty_like(o)
        c = torch.zeros(1, dtype=torch.int32, device="cuda")
        shaded = torch.full((sp.count,), 0x5A5A5A5A, dtype=torch.int32, device="cuda")
        spec = [(sp, view, o.data_ptr(), k.data_ptr(), c.data_ptr())]
        ctx.sort_batch(spec)
        ctx.sync()
        assert torch.all(shaded == 0x5A5A5A5A)
        ctx.sort_batch_shaded(spec, [(eye, shaded.data_ptr())])
        ctx.sync()
        order = o[:int(c.item())].cpu().numpy().view(np.uint32)
        got = shaded.cpu().numpy().view(np.uint32)
        assert np.array_equal(got[order], O.shade(parsed.centers, sh, 3, order, eye))
        shaded.fill_(0x5A5A5A5A)
        ctx.sort_batch(spec)
        ctx.sync()
        assert torch.all(shaded == 0x5A5A5A5A)
    finally:
        sp.destroy()


@pytest.mark.gpu
def test_harmonics_refusals(ctx):
    job = W.uniform_100k(seed=70, n=1000)
    sp = parse_splats(job.records, ctx)
    try:
        with pytest.raises(WsError, match="degree must be 0 to 3"):
            sp.set_harmonics(4, np.zeros(10, np.uint32))
        with pytest.raises(WsError, match="needed"):
            sp.set_harmonics(2, np.zeros(100, np.uint32))
        sp.set_harmonics(1, np.zeros(SH_WORDS[1] * sp.count, np.uint32))
        sp.set_harmonics(0, None)
    finally:
        sp.destroy()
