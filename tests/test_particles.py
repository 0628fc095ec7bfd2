"""The particle sort of alpha emitters (render/particles.js:197-243).

CPU: the oracle against the reference's own case (two particles of one
emitter on the view axis, the near one born first, drawn far first:
test/gpu.test.js:2666-2711) and hand-checked keys; the library's depth
thresholds (host code, no device) against the oracle's bucket function at
and around every threshold and over a log-uniform sweep of depths.
GPU: every emitter of a batch against the oracle, bit for bit, including
particles placed exactly on and just below bucket thresholds, dead and
never-used slots, non-finite positions, empty rings and a large ring.
"""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O
from winding_b200 import WsError, particles as P

CULLED = O.CULLED


def _particle(pos, age=0.0, life=1.0, vel=(0.0, 0.0, 0.0)):
    return np.array([*pos, age, *vel, life], np.float32)


def _pool(rng, n, spread=30.0, dead=0.2):
    pool = np.zeros((n, 8), np.float32)
    pool[:, 0:3] = rng.normal(size=(n, 3)) * spread
    pool[:, 4:7] = rng.normal(size=(n, 3))
    pool[:, 7] = rng.uniform(0.5, 4.0, size=n)
    pool[:, 3] = pool[:, 7] * rng.uniform(0.0, 1.0, size=n)
    dying = rng.random(n) < dead
    pool[dying, 3] = pool[dying, 7] + rng.uniform(0, 1, size=dying.sum())   # age >= lifetime
    never = rng.random(n) < dead / 4
    pool[never, 3] = 0.0
    pool[never, 7] = 0.0                                                     # a slot never used
    return pool


# ------------------------------------------------------------------ CPU

def test_reference_case_far_particle_first():
    # Camera at (0, 0, 5) looking at the origin; the first particle (slot 0)
    # at z = 1 (depth 4), the second (slot 1) at z = -2 (depth 7).
    eye = np.array([0, 0, 5], np.float32)
    fwd = np.array([0, 0, -1], np.float32)
    pool = np.stack([_particle((0, 0, 1), 4.9, 10.0), _particle((0, 0, -2), 0.0, 10.0)])
    order, keys = O.particle_sort(pool, 0, 2, eye, fwd)
    assert list(order) == [1, 0]
    assert keys[0] < keys[1]


def test_keys_by_hand():
    eye = np.zeros(3, np.float32)
    fwd = np.array([0, 0, 1], np.float32)
    # depth 9: log2 9 = 3.1699..., (13.1699 * 4095) / 30 = 1797.7 -> bucket 1797
    assert O.particle_key(_particle((0, 0, 9)), eye, fwd) == 4095 - 1797
    # depth 1: (0 + 10) * 4095 / 30 = 1365 exactly
    assert O.particle_key(_particle((0, 0, 1)), eye, fwd) == 4095 - 1365
    # at and beyond 2^20, and at or below 2^-10, the buckets clamp
    assert O.particle_key(_particle((0, 0, 2.0 ** 20)), eye, fwd) == 0
    assert O.particle_key(_particle((0, 0, 1e30)), eye, fwd) == 0
    assert O.particle_key(_particle((0, 0, np.inf)), eye, fwd) == 0
    assert O.particle_key(_particle((0, 0, 2.0 ** -10)), eye, fwd) == 4095
    assert O.particle_key(_particle((0, 0, -5)), eye, fwd) == 4095      # behind: depth 1e-6
    assert O.particle_key(_particle((np.nan, 0, 5)), eye, fwd) == 4095  # NaN depth: max gives 1e-6
    # dead: age >= lifetime; a slot never used has both 0; NaN age is live
    assert O.particle_key(_particle((0, 0, 9), 1.0, 1.0), eye, fwd) == CULLED
    assert O.particle_key(_particle((0, 0, 9), 0.0, 0.0), eye, fwd) == CULLED
    assert O.particle_key(_particle((0, 0, 9), np.nan, 1.0), eye, fwd) == 4095 - 1797


def test_oracle_sort_is_stable_and_offsets_slots():
    rng = np.random.default_rng(3)
    pool = _pool(rng, 5000, spread=0.01)        # a tight ball: many equal keys
    eye = np.array([0, 0, 40], np.float32)
    fwd = np.array([0, 0, -1], np.float32)
    order, keys = O.particle_sort(pool, 1000, 3000, eye, fwd)
    assert np.all(order >= 1000) and np.all(order < 4000)
    assert np.all(np.diff(keys.astype(np.int64)) >= 0)
    same = keys[1:] == keys[:-1]
    assert np.all(order[1:][same] > order[:-1][same])
    want = [i for i in range(1000, 4000) if O.particle_key(pool[i], eye, fwd) != CULLED]
    assert sorted(order.tolist()) == want


def _oracle_bucket(d):
    k = O.particle_key(_particle((0, 0, d)), np.zeros(3, np.float32), np.array([0, 0, 1], np.float32))
    return 4095 - k


def test_library_thresholds_agree_with_the_oracle():
    thr = P.thresholds()
    assert thr[0] == 0 and np.all(np.diff(thr.astype(np.float64)) >= 0)
    probe = []
    bits = thr[1:].view(np.uint32).astype(np.int64)
    for off in (-2, -1, 0, 1, 2):
        probe.append((bits + off).astype(np.uint32).view(np.float32))
    rng = np.random.default_rng(5)
    probe.append(np.exp2(rng.uniform(-12, 22, size=20000)).astype(np.float32))
    probe.append(np.array([1e-6, 2.0 ** -10, 1.0, 2.0 ** 20, 3e38, np.inf], np.float32))
    d = np.concatenate(probe)
    d = d[d >= np.float32(1e-6)]
    by_table = np.searchsorted(thr[1:], d, side="right")        # buckets b >= 1 with thr[b] <= d
    for x, b in zip(d[::7], by_table[::7]):                     # the oracle is a per-call ctypes loop
        assert _oracle_bucket(x) == b, (x, b)
    for x, b in zip(d[: 5 * 4095], by_table[: 5 * 4095]):       # every threshold and its neighbours
        assert _oracle_bucket(x) == b, (x, b)


# ------------------------------------------------------------------ GPU

def _device_rings(ctx, pool, rings, eye, fwd):
    import torch
    dev_pool = torch.from_numpy(pool.reshape(-1).copy()).cuda()
    outs = []
    for off, cap in rings:
        n = max(cap, 1)
        outs.append((torch.full((n,), -1, dtype=torch.int32, device="cuda"),
                     torch.full((n,), -1, dtype=torch.int32, device="cuda"),
                     torch.zeros(1, dtype=torch.int32, device="cuda")))
    P.sort_emitters(ctx, dev_pool.data_ptr(), rings, eye, fwd,
                    [(o.data_ptr(), k.data_ptr(), c.data_ptr()) for o, k, c in outs])
    ctx.sync()
    res = []
    for o, k, c in outs:
        s = int(c.item())
        res.append((o[:s].cpu().numpy().view(np.uint32), k[:s].cpu().numpy().view(np.uint32)))
    return res, dev_pool


def _check(ctx, pool, rings, eye, fwd):
    got, _ = _device_rings(ctx, pool, rings, eye, fwd)
    for (off, cap), (o, k) in zip(rings, got):
        want_o, want_k = O.particle_sort(pool, off, cap, eye, fwd)
        assert np.array_equal(o, want_o), (off, cap)
        assert np.array_equal(k, want_k), (off, cap)


@pytest.mark.gpu
def test_reference_case_on_gpu(ctx):
    eye = np.array([0, 0, 5], np.float32)
    fwd = np.array([0, 0, -1], np.float32)
    pool = np.stack([_particle((0, 0, 1), 4.9, 10.0), _particle((0, 0, -2), 0.0, 10.0)])
    got, _ = _device_rings(ctx, pool, [(0, 2)], eye, fwd)
    assert list(got[0][0]) == [1, 0]


@pytest.mark.gpu
def test_emitter_batch_matches_oracle(ctx):
    rng = np.random.default_rng(11)
    pool = _pool(rng, 400_000)
    rings = [(0, 1000), (1000, 64), (1064, 0), (1064, 150_000), (151_064, 7), (151_071, 248_929)]
    for eye, fwd in [(np.array([0, 0, 60], np.float32), np.array([0, 0, -1], np.float32)),
                     (np.array([13.5, -2.25, 7.0], np.float32),
                      (np.array([-0.48, 0.6, -0.64], np.float32)))]:
        _check(ctx, pool, rings, eye, fwd)


@pytest.mark.gpu
def test_bench_workload_particles_64(ctx):
    """The bench's particle workload, whole: 64 rings of 1k-200k slots in one
    pool, sorted in one launch, every ring against the oracle."""
    from winding_b200 import workloads as W
    rings = W.emitter_rings()
    pool = W.particle_pool(sum(c for _, c in rings))
    _check(ctx, pool, rings, np.array([0.0, 5.0, 80.0], np.float32), np.array([0.0, -0.0624, -0.998], np.float32))


@pytest.mark.gpu
def test_depths_on_bucket_thresholds(ctx):
    """Particles exactly on each threshold and one ulp below: the buckets
    the comparisons give are the oracle's."""
    thr = P.thresholds()
    bits = thr[1:].view(np.uint32).astype(np.int64)
    z = np.concatenate([thr[1:], (bits - 1).astype(np.uint32).view(np.float32),
                        (bits + 1).astype(np.uint32).view(np.float32),
                        np.array([1e-6, 2.0 ** -10, 2.0 ** 20, 3e38, np.inf, -1.0, np.nan], np.float32)])
    pool = np.zeros((z.size, 8), np.float32)
    pool[:, 2] = z
    pool[:, 7] = 1.0
    eye = np.zeros(3, np.float32)
    fwd = np.array([0, 0, 1], np.float32)
    _check(ctx, pool, [(0, z.size)], eye, fwd)


@pytest.mark.gpu
def test_all_dead_and_non_finite(ctx):
    rng = np.random.default_rng(12)
    pool = _pool(rng, 20_000)
    pool[:5000, 3] = pool[:5000, 7]                         # ring 0: all dead
    pool[5000:6000, 0] = np.nan                             # NaN positions
    pool[6000:7000, 2] = np.inf
    pool[7000:8000, 3] = np.nan                             # NaN age: live
    eye = np.array([1, 2, 3], np.float32)
    fwd = np.array([0.6, 0, 0.8], np.float32)
    _check(ctx, pool, [(0, 5000), (5000, 15_000)], eye, fwd)
    got, _ = _device_rings(ctx, pool, [(0, 5000)], eye, fwd)
    assert got[0][0].size == 0


@pytest.mark.gpu
def test_large_ring_properties(ctx):
    rng = np.random.default_rng(13)
    n = 3_000_000
    pool = _pool(rng, n, spread=200.0)
    eye = np.array([0, 0, 500], np.float32)
    fwd = np.array([0, 0, -1], np.float32)
    got, _ = _device_rings(ctx, pool, [(0, n)], eye, fwd)
    o, k = got[0]
    assert np.all(np.diff(k.astype(np.int64)) >= 0)
    same = k[1:] == k[:-1]
    assert np.all(o[1:][same] > o[:-1][same])
    want_o, want_k = O.particle_sort(pool, 0, n, eye, fwd)
    assert np.array_equal(o, want_o) and np.array_equal(k, want_k)


@pytest.mark.gpu
def test_refusals(ctx):
    import torch
    pool = torch.zeros(64, dtype=torch.float32, device="cuda")
    o = torch.zeros(8, dtype=torch.int32, device="cuda")
    c = torch.zeros(1, dtype=torch.int32, device="cuda")
    eye, fwd = np.zeros(3, np.float32), np.array([0, 0, 1], np.float32)
    with pytest.raises(WsError, match="16-byte aligned"):
        ctx.sort_particles([(pool.data_ptr() + 4, 0, 1, eye, fwd, o.data_ptr(), None, c.data_ptr())])
    with pytest.raises(WsError, match="needs a pool"):
        ctx.sort_particles([(pool.data_ptr(), 0, 1, eye, fwd, 0, None, c.data_ptr())])
    with pytest.raises(WsError, match="past slot"):
        ctx.sort_particles([(pool.data_ptr(), 0xFFFFFFF0, 0x20, eye, fwd, o.data_ptr(), None, c.data_ptr())])
    ctx.sort_particles([])
