"""Sharding of sort jobs and resident scenes across ranks.

CPU: the plan (every job once, balanced, identical on every rank), scene
placement with hot-scene replicas, and two gloo ranks that each sort only
their share and gather the per-job results on rank 0 (the oracle stands in
for the GPU sort there; what is tested is the host-side split). GPU: two
ranks' shares sorted one after the other on one device through the batched
entry point, checked job by job against the plain sort.
"""
import os
import tempfile
import zlib

import numpy as np
import pytest

from winding_b200 import shard


def test_assign_covers_every_job_once():
    rng = np.random.default_rng(0)
    for world in (1, 2, 3, 8):
        sizes = rng.integers(0, 1000, size=37).tolist()
        plan = shard.assign_jobs(sizes, world)
        assert len(plan) == world
        flat = sorted(i for lst in plan for i in lst)
        assert flat == list(range(37))
        for lst in plan:
            assert lst == sorted(lst)


def test_assign_is_deterministic_and_balanced():
    rng = np.random.default_rng(1)
    sizes = np.exp(rng.uniform(np.log(1e4), np.log(2e6), size=64)).astype(int).tolist()
    for world in (2, 4, 8):
        a = shard.assign_jobs(sizes, world)
        b = shard.assign_jobs(list(sizes), world)
        assert a == b
        ld = shard.loads(a, sizes)
        # Graham's LPT bound against the trivial lower bound of the optimum.
        opt_lb = max(sum(sizes) / world, max(sizes))
        assert max(ld) <= 4 / 3 * opt_lb + 1


def test_assign_edges():
    assert shard.assign_jobs([], 3) == [[], [], []]
    assert shard.assign_jobs([5, 5], 4) == [[0], [1], [], []]
    assert shard.assign_jobs([0, 0, 0], 2) == [[0, 2], [1]]
    with pytest.raises(ValueError):
        shard.assign_jobs([1], 0)
    with pytest.raises(ValueError):
        shard.assign_jobs([-1], 1)
    with pytest.raises(ValueError):
        shard.my_jobs([1, 2], 2, 2)


def test_place_scenes_replicates_hot_scene():
    sizes = [1_000_000, 200_000, 200_000, 200_000]
    rates = [50.0, 1.0, 1.0, 1.0]
    pl = shard.place_scenes(sizes, 4, rates)
    assert len(pl.ranks[0]) > 1            # the hot scene lives on several ranks
    for s in range(1, 4):
        assert len(pl.ranks[s]) == 1
    seen = {pl.route(0, t) for t in range(8)}
    assert seen == set(pl.ranks[0])
    for r in range(4):
        for s in pl.scenes_on(r):
            assert r in pl.ranks[s]


def test_place_scenes_memory():
    sizes = [1000, 1000, 1000]
    with pytest.raises(ValueError):
        shard.place_scenes(sizes, 1, memory_per_rank=1000 * 41 * 2)
    pl = shard.place_scenes(sizes, 3, rates=[100.0, 1.0, 1.0], memory_per_rank=1000 * 41)
    assert all(len(h) == 1 for h in pl.ranks)   # no room for a copy anywhere


def _jobs(seed=7, count=6):
    from winding_b200 import workloads as W
    rng = np.random.default_rng(seed)
    out = []
    for j in range(count):
        n = int(rng.integers(300, 3000))
        rec = W.uniform(n, seed + j) if j % 2 else W.clusters(n, seed + j, k=4, extent=8.0)
        mv = W.random_pose(rng, 15.0, 30.0)
        out.append((rec, mv))
    return out


def _sort_job(rec, mv):
    from oracle import oracle as O
    from winding_b200 import camera
    parsed = O.parse_splat(rec.tobytes())
    proj = camera.perspective(np.pi / 3, 1920 / 1080, 0.1)
    order, keys = O.sort_view(parsed, mv, proj, (1920.0, 1080.0), 0.5)
    return int(len(order)), zlib.crc32(np.asarray(order, np.uint32).tobytes()), \
        zlib.crc32(np.asarray(keys, np.uint32).tobytes())


def _rank_main(rank, world, port, out_path):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        jobs = _jobs()
        sizes = [len(rec) for rec, _ in jobs]
        mine = shard.my_jobs(sizes, rank, world)
        results = {i: _sort_job(*jobs[i]) for i in mine}
        gathered = [None] * world
        dist.all_gather_object(gathered, results)
        if rank == 0:
            merged = {}
            for part in gathered:
                for i, v in part.items():
                    assert i not in merged
                    merged[i] = v
            with open(out_path, "w") as f:
                f.write(repr(sorted(merged.items())))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_sort_their_shares():
    import socket

    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "merged.txt")
        mp.start_processes(_rank_main, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
        merged = dict(eval(open(out).read()))
    jobs = _jobs()
    assert sorted(merged) == list(range(len(jobs)))
    for i, (rec, mv) in enumerate(jobs):
        assert merged[i] == _sort_job(rec, mv)


@pytest.mark.gpu
def test_shares_on_one_gpu_match_plain(ctx):
    """Two ranks' shares of a batch, each sorted in one batched launch (one
    after the other, nothing waiting on the other), give every job the
    plain sort's result."""
    import torch

    from winding_b200 import camera, make_view, parse_splats
    jobs = _jobs(seed=11, count=9)
    proj = camera.perspective(np.pi / 3, 1920 / 1080, 0.1)
    clouds = [parse_splats(rec, ctx) for rec, _ in jobs]
    views = [make_view(mv, proj, (1920, 1080), 0.5) for _, mv in jobs]
    try:
        outs = []
        for sp in clouds:
            n = max(sp.count, 1)
            outs.append((torch.empty(n, dtype=torch.int32, device="cuda"),
                         torch.empty(n, dtype=torch.int32, device="cuda"),
                         torch.zeros(1, dtype=torch.int32, device="cuda")))
        plan = shard.assign_jobs([sp.count for sp in clouds], 2)
        for rank in range(2):
            specs = [(clouds[i], views[i], outs[i][0].data_ptr(), outs[i][1].data_ptr(), outs[i][2].data_ptr())
                     for i in plan[rank]]
            ctx.sort_batch(specs)
        ctx.sync()
        for i, sp in enumerate(clouds):
            order, keys = ctx.sort(sp, views[i])
            c = int(outs[i][2].item())
            assert c == len(order)
            assert np.array_equal(outs[i][0][:c].cpu().numpy().view(np.uint32), order)
            assert np.array_equal(outs[i][1][:c].cpu().numpy().view(np.uint32), keys)
    finally:
        for sp in clouds:
            sp.destroy()
