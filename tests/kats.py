"""Known-answer inputs restated from the reference's own tests.

Each builder cites the reference test (paths in the reference project) whose
inputs and expected outcome it restates. Shared by the oracle tests (CPU) and
the GPU parity tests.
"""
import math
import struct

import numpy as np


def splat_record(pos, scale, rgba, rot) -> bytes:
    """One .splat record: test/splats.test.js:22-30."""
    return struct.pack("<6f", *pos, *scale) + bytes(rgba) + bytes(rot)


# test/splats.test.js:51-61: an unturned record.
UNTURNED = splat_record((1, 2, 3), (0.5, 2, 1), (10, 20, 30, 200), (255, 128, 128, 128))
UNTURNED_COV = (0.25, 0.0, 0.0, 4.0, 0.0, 1.0)

# test/splats.test.js:63-71: a quarter turn about z (w = z = cos 45).
_B = 128 + round(math.sqrt(0.5) * 128)
QUARTER = splat_record((0, 0, 0), (0.5, 2, 1), (0, 0, 0, 255), (_B, 128, 128, _B))

# test/splats.test.js:331-348: what is refused, by message.
REFUSED = [
    (bytes(33), "not a whole number of 32-byte"),
    (splat_record((float("nan"), 0, 0), (1, 1, 1), (0, 0, 0, 0), (255, 128, 128, 128)),
     "splat 0 has a position that is not a number"),
    (bytes([0x50, 0x4B, 0x03, 0x04]) + bytes(60), "this is a zip"),
    (bytes([0x1F, 0x8B]) + bytes(62), "this is gzipped"),
]


def two_splats(red_first: bool) -> bytes:
    """test/gpu.test.js:1813-1840: red at z=1, blue at z=-1, opaque, 0.4 wide."""
    red = splat_record((0, 0, 1), (0.4, 0.4, 0.4), (255, 0, 0, 255), (255, 128, 128, 128))
    blue = splat_record((0, 0, -1), (0.4, 0.4, 0.4), (0, 0, 255, 255), (255, 128, 128, 128))
    return red + blue if red_first else blue + red


def speck_file() -> bytes:
    """test/gpu.test.js:1925-1944: a faint speck (0.37 opacity-pixels) and a large opaque splat."""
    def rec(x, scale, alpha):
        return splat_record((x, 0, 0), (scale, scale, scale), (255, 255, 255, alpha), (255, 128, 128, 128))
    return rec(0, 0.0005, 50) + rec(1, 0.2, 255)


def gpu_test_camera(z: float):
    """The GPU suite's camera: Camera({fovY: 0.8, near: 0.1}) at (0, 0, z)
    looking at the origin, on a 160 x 120 canvas (test/gpu.test.js:1836-1838)."""
    from winding_b200.camera import look_at, perspective
    return look_at((0, 0, z), (0, 0, 0)), perspective(0.8, 160 / 120, 0.1), (160.0, 120.0)


def lcg_keys(n: int = 2000, seed: int = 12345):
    """test/render.test.js:407-426: seed = (seed * 1103515245 + 12345) >>> 0,
    evaluated in doubles as JavaScript does before ToUint32."""
    keys = []
    for _ in range(n):
        seed = int(float(seed) * 1103515245.0 + 12345.0) % (1 << 32)
        keys.append(seed)
    return keys


def scattered_keys(n: int = 500):
    """test/render.test.js:388-405: (i * 2654435761) >>> 8, in doubles."""
    return [int(float(i) * 2654435761.0) % (1 << 32) >> 8 for i in range(n)]


STABLE_PAIRS = [(7, 0), (3, 1), (7, 2), (3, 3), (7, 4), (1, 5)]   # render.test.js:428-438
STABLE_KEYS = [1, 3, 3, 7, 7, 7]
STABLE_PAYLOADS = [5, 1, 3, 0, 2, 4]
SKIPPED_PASS = [40, 10, 30, 20, 50]                                # render.test.js:440-448
