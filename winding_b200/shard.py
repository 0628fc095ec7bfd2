"""Partitioning sort work across GPUs: one process per GPU, no collective on
the data path.

Every (cloud, view) job is independent -- the reference sorts each cloud of a
frame with its own three dispatches (src/render/splats.js:676-697) and no
cloud's order depends on another's -- so several GPUs split a batch by job
and a serving fleet splits by resident scene. Each rank sorts only its own
share, on its own device, into its own outputs; nothing is exchanged. A
collective appears only where a caller wants a summary on one rank (the
survivor counts, for instance), and never between the kernels.

A single cloud is not split: its stable order needs every splat's key
before any position is final, so N GPUs on one cloud run as N replicas.

    plan = assign_jobs([sp.count for sp in clouds], world)
    mine = plan[rank]                     # job indices this rank sorts
    ctx.sort_batch([specs[i] for i in mine], stream)
"""
from __future__ import annotations

import heapq
from dataclasses import dataclass


def assign_jobs(sizes, world: int) -> list[list[int]]:
    """Longest-processing-time-first assignment of jobs to `world` ranks.

    Jobs are taken largest first (ties by index) and each goes to the rank
    with the least work so far (ties by fewer jobs, then by rank: an empty
    cloud still costs a launch's fixed work), so every rank computes the same
    plan from the same sizes without talking to the others. Each rank's list
    is in ascending job order. The largest rank load is at most 4/3 of the
    optimum (Graham's bound) plus nothing for jobs of equal size."""
    if world < 1:
        raise ValueError(f"world must be 1 or more, got {world}")
    sizes = [int(s) for s in sizes]
    if any(s < 0 for s in sizes):
        raise ValueError("job sizes must be 0 or more")
    order = sorted(range(len(sizes)), key=lambda i: (-sizes[i], i))
    heap = [(0, 0, r) for r in range(world)]
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, count, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + sizes[i], count + 1, r))
    for lst in out:
        lst.sort()
    return out


def loads(plan: list[list[int]], sizes) -> list[int]:
    """Total size per rank of a plan."""
    return [sum(int(sizes[i]) for i in lst) for lst in plan]


@dataclass(frozen=True)
class Placement:
    """Where each resident scene lives: scene -> ranks holding a copy."""
    ranks: tuple[tuple[int, ...], ...]

    def route(self, scene: int, ticket: int) -> int:
        """The rank that serves request `ticket` for `scene`: its copies in
        turn, so a replicated scene's requests alternate between them."""
        holders = self.ranks[scene]
        return holders[ticket % len(holders)]

    def scenes_on(self, rank: int) -> list[int]:
        return [s for s, holders in enumerate(self.ranks) if rank in holders]


def place_scenes(sizes, world: int, rates=None, memory_per_rank: int | None = None,
                 bytes_per_splat: int = 41) -> Placement:
    """Places resident scenes on ranks for serving.

    Each scene goes to one rank by expected load (splats x request rate,
    largest first, least-loaded rank). A scene whose load exceeds the mean
    per-rank load is then copied to further ranks (least loaded first,
    memory allowing) until each copy's share is at or below that mean: hot
    scenes are replicated, cold ones live once. `bytes_per_splat` is the
    device footprint of a resident splat (16-byte centre, 24-byte covariance
    and the 1-byte covariance exponent).
    """
    n = len(sizes)
    rates = [1.0] * n if rates is None else [float(r) for r in rates]
    if len(rates) != n:
        raise ValueError("one rate per scene")
    weight = [int(s) * r for s, r in zip(sizes, rates)]
    plan = assign_jobs([int(w) for w in weight], world)
    holders = [[r] for r in range(n)]
    for r, lst in enumerate(plan):
        for s in lst:
            holders[s] = [r]
    mem = [0] * world
    for s in range(n):
        mem[holders[s][0]] += int(sizes[s]) * bytes_per_splat
    if memory_per_rank is not None and max(mem, default=0) > memory_per_rank:
        raise ValueError("the scenes do not fit in the ranks' memory")
    load = [0.0] * world
    for s in range(n):
        load[holders[s][0]] += weight[s]
    mean = sum(weight) / world if world else 0.0
    for s in sorted(range(n), key=lambda i: (-weight[i], i)):
        while weight[s] / len(holders[s]) > mean and len(holders[s]) < world:
            cands = [r for r in range(world) if r not in holders[s]
                     and (memory_per_rank is None or mem[r] + int(sizes[s]) * bytes_per_splat <= memory_per_rank)]
            if not cands:
                break
            r = min(cands, key=lambda q: (load[q], q))
            share_old = weight[s] / len(holders[s])
            holders[s].append(r)
            share_new = weight[s] / len(holders[s])
            for q in holders[s][:-1]:
                load[q] -= share_old - share_new
            load[r] += share_new
            mem[r] += int(sizes[s]) * bytes_per_splat
    return Placement(tuple(tuple(sorted(h)) for h in holders))


def my_jobs(sizes, rank: int, world: int) -> list[int]:
    """This rank's share of a batch (assign_jobs, evaluated locally)."""
    if not 0 <= rank < world:
        raise ValueError(f"rank {rank} is not in [0, {world})")
    return assign_jobs(sizes, world)[rank]
