"""Seeded synthetic splat clouds and views for the parity tests and the bench.

No capture dataset ships with this library; these generators stand in for
one, with the shapes and value distributions of the five workloads the sort
is measured on:

  uniform-100k    100,000 splats, positions U[-10,10]^3, one camera at 25
  clusters-1M     1,000,000 splats from 32 isotropic Gaussian clusters
                  (centres U[-50,50]^3, sigma U[0.5,5]), camera framing it
  slab-6M         6,000,000 splats in a slab N(0,1)*(40,40,0.8) 100 units in
                  front of the camera, plus 0.1% "frame" splats spread in
                  depth over 50x the slab's +-3 sigma thickness, so ~99.9% of
                  the survivors share ~1300 of the 65536 keys
  mixed-64        64 (scene, view) jobs, counts log-uniform in [10k, 2M],
                  cluster / slab / uniform in turn, cameras on spheres of
                  radius U[20,60] looking at the origin
  served-16       16 resident scenes of 50k-4M splats and a Poisson request
                  stream of random poses

Every splat record is the 32-byte .splat layout (scene/splats.js:14-15 in the
reference): position 3 x f32, scale 3 x f32 (log-normal, mu -4, sigma 0.5),
RGBA 4 x u8 uniform, rotation 4 x u8 = round(128 + 127 q) for a normalised
N(0,1)^4 quaternion q (w, x, y, z). Viewport 1920 x 1080, fovY pi/3, near 0.1.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .camera import Camera, bounds_radius, fit_distance, perspective, look_at

VIEWPORT = (1920.0, 1080.0)
FOV_Y = math.pi / 3
NEAR = 0.1
ASPECT = VIEWPORT[0] / VIEWPORT[1]

RECORD = np.dtype([("pos", "<f4", 3), ("scale", "<f4", 3), ("rgba", "u1", 4), ("rot", "u1", 4)])


@dataclass
class View:
    """What a caller writes into the reference's Cloud uniform for one sort."""
    model_view: np.ndarray      # f32[16], column-major
    projection: np.ndarray      # f32[16]
    viewport: tuple = VIEWPORT
    cull: float = 0.5


@dataclass
class Job:
    """One (cloud, view): the records and the view to sort them for."""
    records: np.ndarray         # RECORD[n]
    view: View
    kind: str = ""

    @property
    def count(self) -> int:
        return int(self.records.shape[0])

    def bytes(self) -> bytes:
        return self.records.tobytes()


def records_from(pos: np.ndarray, rng: np.random.Generator) -> np.ndarray:
    """Complete records around the given positions: scale, colour, rotation."""
    n = pos.shape[0]
    rec = np.empty(n, RECORD)
    rec["pos"] = pos.astype(np.float32)
    rec["scale"] = np.exp(rng.normal(-4.0, 0.5, size=(n, 3))).astype(np.float32)
    rec["rgba"] = rng.integers(0, 256, size=(n, 4), dtype=np.uint8)
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    rec["rot"] = np.clip(np.rint(128 + 127 * q), 0, 255).astype(np.uint8)
    return rec


def _bounds(rec: np.ndarray):
    p = rec["pos"].astype(np.float64)
    return p.min(axis=0), p.max(axis=0)


def _framing_view(rec: np.ndarray, cull: float) -> View:
    """A camera on +z of the cloud's box centre at fitDistance of its radius."""
    lo, hi = _bounds(rec)
    centre = (lo + hi) / 2
    dist = fit_distance(bounds_radius(lo, hi), FOV_Y, ASPECT, 1.0, NEAR)
    cam = Camera(FOV_Y, NEAR)
    cam.position = np.array([centre[0], centre[1], centre[2] + dist], np.float32)
    cam.target = centre.astype(np.float32)
    cam.update(ASPECT)
    return View(cam.view, cam.projection, VIEWPORT, cull)


def uniform(n: int, seed: int, half: float = 10.0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return records_from(rng.uniform(-half, half, size=(n, 3)), rng)


def clusters(n: int, seed: int, k: int = 32, extent: float = 50.0, sigma=(0.5, 5.0)) -> np.ndarray:
    rng = np.random.default_rng(seed)
    centres = rng.uniform(-extent, extent, size=(k, 3))
    sig = rng.uniform(sigma[0], sigma[1], size=k)
    which = rng.integers(0, k, size=n)
    pos = centres[which] + rng.normal(size=(n, 3)) * sig[which, None]
    return records_from(pos, rng)


def slab(n: int, seed: int, spread=(40.0, 40.0, 0.8), depth: float = 100.0,
         frame_fraction: float = 0.001) -> tuple[np.ndarray, View]:
    """The heavy-collision slab, seen from a camera at the origin looking down -z."""
    rng = np.random.default_rng(seed)
    nf = max(1, int(round(n * frame_fraction)))
    ns = n - nf
    pos = np.empty((n, 3))
    pos[:ns] = rng.normal(size=(ns, 3)) * np.asarray(spread)
    pos[:ns, 2] -= depth
    # Frame splats: depth uniform over 50x the slab's 6-sigma thickness,
    # centred on the slab but kept in front of the near plane, inside the view.
    span = 50 * 6 * spread[2]
    d = rng.uniform(max(depth - span / 2, 1.0), depth + span / 2, size=nf)
    ty = math.tan(FOV_Y / 2)
    pos[ns:, 0] = rng.uniform(-0.9, 0.9, size=nf) * ty * ASPECT * d
    pos[ns:, 1] = rng.uniform(-0.9, 0.9, size=nf) * ty * d
    pos[ns:, 2] = -d
    perm = rng.permutation(n)
    rec = records_from(pos[perm], rng)
    view = View(look_at((0, 0, 0), (0, 0, -1)), perspective(FOV_Y, ASPECT, NEAR), VIEWPORT, 0.5)
    return rec, view


def uniform_100k(seed: int = 0, cull: float = 0.5, n: int = 100_000) -> Job:
    rec = uniform(n, seed)
    cam = Camera(FOV_Y, NEAR)
    cam.position = np.array([0, 0, 25], np.float32)
    cam.update(ASPECT)
    return Job(rec, View(cam.view, cam.projection, VIEWPORT, cull), "uniform")


def clusters_1m(seed: int = 1, cull: float = 0.5, n: int = 1_000_000) -> Job:
    rec = clusters(n, seed)
    return Job(rec, _framing_view(rec, cull), "clusters")


def slab_6m(seed: int = 2, cull: float = 0.5, n: int = 6_000_000) -> Job:
    rec, view = slab(n, seed)
    view.cull = cull
    return Job(rec, view, "slab")


def random_pose(rng: np.random.Generator, rmin: float = 20.0, rmax: float = 60.0) -> np.ndarray:
    """A view matrix from a point on a sphere of radius U[rmin, rmax] looking
    at the origin, rejecting directions within 0.99 of the up axis."""
    while True:
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        if abs(d[1]) <= 0.99:
            break
    r = rng.uniform(rmin, rmax)
    return look_at(d * r, (0, 0, 0))


def scene(kind: str, n: int, seed: int) -> np.ndarray:
    """A scene of `n` splats that fits a +-10 box: cluster, slab or uniform."""
    if kind == "cluster":
        return clusters(n, seed, k=8, extent=8.0, sigma=(0.3, 2.0))
    if kind == "slab":
        rng = np.random.default_rng(seed)
        pos = rng.normal(size=(n, 3)) * np.array([4.0, 4.0, 0.08])
        return records_from(pos, rng)
    return uniform(n, seed)


KINDS = ("cluster", "slab", "uniform")


def scaled_counts(rng: np.random.Generator, jobs: int, lo: int, hi: int, total: int) -> np.ndarray:
    """`jobs` counts drawn log-uniform in [lo, hi], then scaled by one common
    factor (each clipped to [lo, hi]) so that they add up to `total`: the
    draw's shape, the workload's stated size."""
    raw = np.exp(rng.uniform(math.log(lo), math.log(hi), size=jobs))
    a, b = 1e-3, 1e3
    for _ in range(200):
        f = math.sqrt(a * b)
        if np.clip(raw * f, lo, hi).sum() < total:
            a = f
        else:
            b = f
    counts = np.clip(np.floor(raw * math.sqrt(a * b)), lo, hi).astype(np.int64)
    counts[int(np.argmin(counts))] += total - int(counts.sum())   # the rounding remainder, on the smallest job
    return counts


def mixed_64(seed: int = 3, jobs: int = 64, lo: int = 10_000, hi: int = 2_000_000,
             cull: float = 0.5, total: int = 25_000_000) -> list[Job]:
    """64 (scene, view) jobs of about 25M splats in all: counts log-uniform in
    [10k, 2M] scaled to the total, scenes cycling cluster / slab / uniform,
    cameras on spheres of radius 20-60 looking at the origin."""
    rng = np.random.default_rng(seed)
    counts = scaled_counts(rng, jobs, lo, hi, total)
    proj = perspective(FOV_Y, ASPECT, NEAR)
    out = []
    for j in range(jobs):
        kind = KINDS[j % 3]
        rec = scene(kind, int(counts[j]), seed * 1000 + j)
        out.append(Job(rec, View(random_pose(rng), proj, VIEWPORT, cull), kind))
    return out


def served_16(seed: int = 4, scenes: int = 16, lo: int = 50_000, hi: int = 4_000_000) -> list[np.ndarray]:
    rng = np.random.default_rng(seed)
    counts = np.exp(rng.uniform(math.log(lo), math.log(hi), size=scenes)).astype(np.int64)
    return [scene(KINDS[j % 3], int(counts[j]), seed * 1000 + j) for j in range(scenes)]


def poisson_arrivals(rate_hz: float, duration_s: float, seed: int = 5) -> np.ndarray:
    """Arrival times (seconds) of a Poisson stream."""
    rng = np.random.default_rng(seed)
    n = int(rate_hz * duration_s * 1.5) + 16
    t = np.cumsum(rng.exponential(1.0 / rate_hz, size=n))
    return t[t < duration_s]


# ----------------------------------------------------------------- particles

def particle_pool(n: int, seed: int = 7, spread: float = 20.0, dead: float = 0.15) -> np.ndarray:
    """A pool of n 32-byte particles (position, age, velocity, lifetime as
    f32; render/particles.js:51-56): positions N(0, spread), lifetimes
    U[0.5, 4] s, a `dead` share past their lifetime and some never used."""
    rng = np.random.default_rng(seed)
    pool = np.zeros((n, 8), np.float32)
    pool[:, 0:3] = rng.normal(size=(n, 3)) * spread
    pool[:, 4:7] = rng.normal(size=(n, 3))
    pool[:, 7] = rng.uniform(0.5, 4.0, size=n)
    pool[:, 3] = pool[:, 7] * rng.uniform(0.0, 1.0, size=n)
    gone = rng.random(n) < dead
    pool[gone, 3] = pool[gone, 7] + 0.1
    return pool


def emitter_rings(emitters: int = 64, lo: int = 1_000, hi: int = 200_000, seed: int = 8) -> list[tuple[int, int]]:
    """(offset, capacity) of `emitters` rings laid end to end in one pool,
    capacities log-uniform in [lo, hi]."""
    rng = np.random.default_rng(seed)
    caps = np.exp(rng.uniform(math.log(lo), math.log(hi), size=emitters)).astype(np.int64)
    offs = np.concatenate([[0], np.cumsum(caps)[:-1]])
    return [(int(o), int(c)) for o, c in zip(offs, caps)]


# ----------------------------------------------------------------- harmonics and .ply

SH_COEFFICIENTS = (0, 3, 8, 15)


def harmonics_words(n: int, degree: int, seed: int = 9, scale: float = 0.3) -> np.ndarray:
    """Random harmonics of `degree` for n splats, packed as the reference
    packs them (ceil(3 c / 2) words a splat of half floats, scene/splats.js:306-333)."""
    rng = np.random.default_rng(seed)
    c = SH_COEFFICIENTS[degree]
    per = (3 * c + 1) // 2
    halves = np.zeros((n, per * 2), np.float16)
    halves[:, :3 * c] = rng.uniform(-scale, scale, size=(n, 3 * c)).astype(np.float16)
    return halves.view(np.uint16).reshape(-1).view(np.uint32).copy()


def ply_bytes(n: int, degree: int = 0, seed: int = 10) -> bytes:
    """A binary .ply as training writes it (scene/splats.js:6-13): x y z,
    normals, f_dc_0..2, opacity, scale_0..2, rot_0..3 and 9, 24 or 45
    f_rest_ properties, all float."""
    rng = np.random.default_rng(seed)
    rest = 3 * SH_COEFFICIENTS[degree]
    names = ["x", "y", "z", "nx", "ny", "nz", "f_dc_0", "f_dc_1", "f_dc_2", "opacity",
             "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3"] + [f"f_rest_{k}" for k in range(rest)]
    cols = np.zeros((n, len(names)), np.float32)
    cols[:, 0:3] = rng.normal(0, 10, (n, 3))
    cols[:, 6:9] = rng.normal(0, 1.5, (n, 3))
    cols[:, 9] = rng.normal(0, 4, n)
    cols[:, 10:13] = rng.normal(-4, 1, (n, 3))
    cols[:, 13:17] = rng.normal(size=(n, 4))
    cols[:, 17:] = rng.normal(0, 0.3, (n, rest))
    head = ("ply\nformat binary_little_endian 1.0\nelement vertex %d\n" % n
            + "".join(f"property float {p}\n" for p in names) + "end_header\n").encode()
    return head + cols.astype("<f4").tobytes()
