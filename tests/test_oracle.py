"""The CPU oracle against the reference's known answers, a second
restatement, and the committed golden fixtures. No GPU needed."""
import glob
import os

import numpy as np
import pytest

from oracle import oracle as O
from oracle import pyoracle as P
from tests import kats
from winding_b200 import workloads as W

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_unturned_record_decodes_to_its_scales_squared():
    s = O.parse_splat(kats.UNTURNED)
    assert s.count == 1
    assert list(s.centers[0, :3]) == [1, 2, 3]
    assert list(s.colours.view(np.uint8).reshape(-1, 4)[0]) == [10, 20, 30, 200]
    assert np.allclose(s.covariances[0], kats.UNTURNED_COV, atol=1e-4)
    assert list(s.min) == [1, 2, 3] and list(s.max) == [1, 2, 3]


def test_quarter_turn_moves_the_long_axis():
    s = O.parse_splat(kats.QUARTER)
    xx, xy, _, yy = s.covariances[0, :4]
    assert abs(xx - 4) <= 1e-2 and abs(yy - 0.25) <= 1e-2 and abs(xy) <= 1e-2


@pytest.mark.parametrize("data,message", kats.REFUSED)
def test_refusals_by_message(data, message):
    with pytest.raises(O.OracleError, match=message):
        O.parse_splat(data)


def test_drawlist_stability():
    k, p = O.drawlist_sort([k for k, _ in kats.STABLE_PAIRS], [p for _, p in kats.STABLE_PAIRS])
    assert list(k) == kats.STABLE_KEYS and list(p) == kats.STABLE_PAYLOADS


def test_drawlist_against_a_reference_sort():
    keys = kats.lcg_keys()
    k, p = O.drawlist_sort(keys, list(range(len(keys))))
    want = sorted(range(len(keys)), key=lambda i: keys[i])
    assert list(p) == want and list(k) == [keys[i] for i in want]
    s = kats.scattered_keys()
    k, _ = O.drawlist_sort(s, list(range(len(s))))
    assert list(k) == sorted(s)


def test_drawlist_skipped_passes_and_trivial_lists():
    k, p = O.drawlist_sort(kats.SKIPPED_PASS, kats.SKIPPED_PASS)
    assert list(k) == sorted(kats.SKIPPED_PASS) and list(p) == sorted(kats.SKIPPED_PASS)
    k, p = O.drawlist_sort([], [])
    assert k.size == 0
    k, p = O.drawlist_sort([9], [9])
    assert list(k) == [9]


@pytest.mark.parametrize("red_first", [True, False])
def test_two_splats_back_to_front_from_either_side(red_first):
    parsed = O.parse_splat(kats.two_splats(red_first))
    red, blue = (0, 1) if red_first else (1, 0)
    mv, proj, vp = kats.gpu_test_camera(5.0)
    order, keys = O.sort_view(parsed, mv, proj, vp, 0.5)
    assert list(order) == [blue, red] and list(keys) == [0, 65535]
    mv, proj, vp = kats.gpu_test_camera(-5.0)
    order, keys = O.sort_view(parsed, mv, proj, vp, 0.5)
    assert list(order) == [red, blue]


def test_single_splat_spans_no_depth_and_takes_the_nearest_key():
    parsed = O.parse_splat(kats.two_splats(True)[:32])
    mv, proj, vp = kats.gpu_test_camera(5.0)
    visible, dmin, dscale = O.depth_range(mv, parsed.min, parsed.max)
    assert visible and dscale == np.float32(65535 / 1e-6)
    order, keys = O.sort_view(parsed, mv, proj, vp, 0.5)
    assert list(order) == [0] and list(keys) == [65535]


def test_speck_is_culled_at_the_default_and_kept_at_zero():
    parsed = O.parse_splat(kats.speck_file())
    mv, proj, vp = kats.gpu_test_camera(5.0)
    order, _ = O.sort_view(parsed, mv, proj, vp, 0.5)
    assert list(order) == [1]
    order, _ = O.sort_view(parsed, mv, proj, vp, 0.0)
    assert sorted(order) == [0, 1]


def test_cloud_behind_the_camera_sorts_nothing():
    parsed = O.parse_splat(kats.two_splats(True))
    from winding_b200.camera import look_at, perspective
    mv = look_at((0, 0, 5), (0, 0, 10))
    order, _ = O.sort_view(parsed, mv, perspective(0.8, 4 / 3, 0.1), (160, 120), 0.5)
    assert order.size == 0


@pytest.mark.parametrize("cull", [0.0, 0.5, 3.0])
def test_oracle_matches_the_python_restatement(cull):
    job = W.clusters_1m(seed=21, n=1500)
    data = job.bytes()
    parsed = O.parse_splat(data)
    c2, cov2, lo, hi = P.decode(data)
    assert np.array_equal(parsed.centers.view(np.uint32), c2.view(np.uint32))
    assert np.array_equal(parsed.covariances.view(np.uint32), cov2.view(np.uint32))
    assert list(parsed.min) == lo and list(parsed.max) == hi
    o1, k1 = O.sort_view(parsed, job.view.model_view, job.view.projection, job.view.viewport, cull)
    o2, k2 = P.sort_view(data, job.view.model_view, job.view.projection, job.view.viewport, cull)
    assert list(o1) == o2 and list(k1) == k2


@pytest.mark.parametrize("cull", [0.0, 0.5])
def test_python_restatement_on_the_real_capture(cull):
    """The two restatements agree on 1500 records of the real capture (the
    cactus fixture: measured scales and rotations, not sampled ones)."""
    g = np.load(os.path.join(GOLDEN, "cactus_posed_16384.npz"))
    data = g["records"].tobytes()[: 1500 * 32]
    parsed = O.parse_splat(data)
    c2, cov2, lo, hi = P.decode(data)
    assert np.array_equal(parsed.centers.view(np.uint32), c2.view(np.uint32))
    assert np.array_equal(parsed.covariances.view(np.uint32), cov2.view(np.uint32))
    mv, pr, vp = g["model_view"], g["projection"], tuple(g["viewport"])
    o1, k1 = O.sort_view(parsed, mv, pr, vp, cull)
    o2, k2 = P.sort_view(data, mv, pr, vp, cull)
    assert len(o2) > 500 and list(o1) == o2 and list(k1) == k2


def test_counting_sort_is_drawlist_order():
    rng = np.random.default_rng(3)
    keys = rng.integers(0, 400, size=20000).astype(np.uint32)
    keys[rng.random(20000) < 0.2] = O.CULLED
    order, sk = O.counting_sort(keys)
    idx = np.nonzero(keys != O.CULLED)[0].astype(np.uint32)
    k, p = O.drawlist_sort(keys[idx], idx)
    assert np.array_equal(order, p) and np.array_equal(sk, k)


def test_threaded_oracle_is_identical():
    job = W.slab_6m(seed=5, n=200_000)
    parsed = O.parse_splat(job.bytes())
    a = O.sort_view(parsed, job.view.model_view, job.view.projection, job.view.viewport, 0.5, threads=1)
    b = O.sort_view(parsed, job.view.model_view, job.view.projection, job.view.viewport, 0.5, threads=7)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "*.npz"))))
def test_oracle_reproduces_the_golden_fixtures(path):
    g = np.load(path)
    parsed = O.parse_splat(g["records"].tobytes())
    for tag, cull in (("0p0", 0.0), ("0p5", 0.5)):
        order, keys = O.sort_view(parsed, g["model_view"], g["projection"], g["viewport"], cull)
        assert np.array_equal(order, g[f"order_{tag}"]) and np.array_equal(keys, g[f"keys_{tag}"])
