"""Writes the golden fixtures of the parity tests (run from the repo root):

    python tests/golden/make_golden.py [path/to/demo/cactus.splat]

Each case is a small seeded cloud from winding_b200.workloads with one view,
or a seeded subset of the reference's real capture (demo/cactus.splat, a
3D Gaussian Splatting scan by Steam Studio released CC0, read from the path
given as the first argument, the file in a checkout of the reference; without
it those two fixtures are left as they are) with a framing or a posed view;
the expected survivor order and keys come from the CPU oracle (oracle/), which
is itself cross-checked against a second restatement (oracle/pyoracle.py) and
the reference's known-answer tests in tests/test_oracle.py. Stored per case:
the .splat records, the view, and for cull 0 and 0.5 the order and keys.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle  # noqa: E402
from winding_b200 import workloads as W  # noqa: E402

CULLS = (0.0, 0.5)
CACTUS_SUBSET = 16384


def cactus_cases(path):
    """Two seeded subsets of the capture (records kept in file order): one
    seen from +z at the fitted distance, one from a seeded direction."""
    if not path or not os.path.exists(path):
        return
    rec = np.fromfile(path, dtype=W.RECORD)
    for name, seed, posed in (("cactus_front_16384", 21, False), ("cactus_posed_16384", 22, True)):
        rng = np.random.default_rng(seed)
        sub = rec[np.sort(rng.choice(len(rec), CACTUS_SUBSET, replace=False))]
        view = W._framing_view(sub, 0.5)
        if posed:
            lo, hi = W._bounds(sub)
            centre = (lo + hi) / 2
            d = rng.normal(size=3)
            d /= np.linalg.norm(d)
            r = W.fit_distance(W.bounds_radius(lo, hi), W.FOV_Y, W.ASPECT, 1.0, W.NEAR) * rng.uniform(0.6, 1.2)
            view = W.View(W.look_at(centre + d * r, centre), view.projection, view.viewport, view.cull)
        yield name, W.Job(sub, view, "capture")


def cases(capture=None):
    yield "uniform_3000", W.uniform_100k(seed=11, n=3000)
    yield "clusters_3000", W.clusters_1m(seed=12, n=3000)
    yield "slab_4000", W.slab_6m(seed=13, n=4000)
    rng = np.random.default_rng(14)
    rec = W.scene("cluster", 2500, 15)
    yield "posed_2500", W.Job(rec, W.View(W.random_pose(rng), W.perspective(W.FOV_Y, W.ASPECT, W.NEAR)), "cluster")
    yield from cactus_cases(capture)


def main():
    capture = sys.argv[1] if len(sys.argv) > 1 else None
    for name, job in cases(capture):
        parsed = oracle.parse_splat(job.bytes())
        out = {
            "records": np.frombuffer(job.bytes(), np.uint8),
            "model_view": np.asarray(job.view.model_view, np.float32),
            "projection": np.asarray(job.view.projection, np.float32),
            "viewport": np.asarray(job.view.viewport, np.float32),
        }
        for cull in CULLS:
            order, keys = oracle.sort_view(parsed, job.view.model_view, job.view.projection, job.view.viewport, cull)
            tag = str(cull).replace(".", "p")
            out[f"order_{tag}"] = order
            out[f"keys_{tag}"] = keys
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **out)
        print(path, {k: v.shape for k, v in out.items() if k.startswith("order")})


if __name__ == "__main__":
    main()
