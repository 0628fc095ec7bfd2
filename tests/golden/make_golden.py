"""Writes the golden fixtures of the parity tests (run from the repo root):

    python tests/golden/make_golden.py

Each case is a small seeded cloud from winding_b200.workloads with one view;
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


def cases():
    yield "uniform_3000", W.uniform_100k(seed=11, n=3000)
    yield "clusters_3000", W.clusters_1m(seed=12, n=3000)
    yield "slab_4000", W.slab_6m(seed=13, n=4000)
    rng = np.random.default_rng(14)
    rec = W.scene("cluster", 2500, 15)
    yield "posed_2500", W.Job(rec, W.View(W.random_pose(rng), W.perspective(W.FOV_Y, W.ASPECT, W.NEAR)), "cluster")


def main():
    for name, job in cases():
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
