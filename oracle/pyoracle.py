"""A second, pure-Python restatement of the same path, for small inputs.

TEST INFRASTRUCTURE ONLY. It exists to cross-check the C++ oracle: every f32
operation here is a numpy float32 scalar op (one IEEE rounding each), every
double operation a Python float op, in the order the reference writes them.
It is slow (a few thousand splats a second) and only used on small cases.

Follows, in the reference project:
  decode + covariance   src/scene/splats.js:335-388
  depth range           src/render/splats.js:559-587
  footprint             src/render/splats.js:102-124
  makeKeys              src/render/splats.js:155-186
  stable order          src/render/drawlist.js:186-229
"""
from __future__ import annotations

import math
import struct

import numpy as np

F = np.float32
BUCKETS = 65536
CULLED = 0xFFFFFFFF


def v8_hypot(*args: float) -> float:
    """Math.hypot as V8 computes it: scaled by the largest magnitude,
    squares summed with Kahan compensation."""
    vals = [abs(a) for a in args]
    m = max(vals)
    if m == 0:
        return 0.0
    s = 0.0
    comp = 0.0
    for a in vals:
        n = a / m
        summand = n * n - comp
        prelim = s + summand
        comp = (prelim - s) - summand
        s = prelim
    return math.sqrt(s) * m


def decode(data: bytes):
    """(centers f32[n,4], cov f32[n,6], min[3], max[3]) from .splat bytes."""
    n = len(data) // 32
    centers = np.zeros((n, 4), np.float32)
    cov = np.zeros((n, 6), np.float32)
    lo = [math.inf] * 3
    hi = [-math.inf] * 3
    for i in range(n):
        rec = data[i * 32:(i + 1) * 32]
        x, y, z, sx, sy, sz = struct.unpack("<6f", rec[:24])
        if not all(math.isfinite(v) for v in (x, y, z)):
            raise ValueError(f"splats: splat {i} has a position that is not a number")
        centers[i, :3] = (x, y, z)
        centers.view(np.uint32)[i, 3] = struct.unpack("<I", rec[24:28])[0]
        for k, p in enumerate((x, y, z)):
            if p < lo[k]:
                lo[k] = p
            if p > hi[k]:
                hi[k] = p
        qw, qx, qy, qz = ((b - 128) / 128 for b in rec[28:32])
        length = v8_hypot(qw, qx, qy, qz) or 1.0
        w, u, v, t = qw / length, qx / length, qy / length, qz / length
        r00 = 1 - 2 * (v * v + t * t); r01 = 2 * (u * v - w * t); r02 = 2 * (u * t + w * v)
        r10 = 2 * (u * v + w * t); r11 = 1 - 2 * (u * u + t * t); r12 = 2 * (v * t - w * u)
        r20 = 2 * (u * t - w * v); r21 = 2 * (v * t + w * u); r22 = 1 - 2 * (u * u + v * v)
        m00, m01, m02 = r00 * sx, r01 * sy, r02 * sz
        m10, m11, m12 = r10 * sx, r11 * sy, r12 * sz
        m20, m21, m22 = r20 * sx, r21 * sy, r22 * sz
        cov[i] = (m00 * m00 + m01 * m01 + m02 * m02, m00 * m10 + m01 * m11 + m02 * m12,
                  m00 * m20 + m01 * m21 + m02 * m22, m10 * m10 + m11 * m11 + m12 * m12,
                  m10 * m20 + m11 * m21 + m12 * m22, m20 * m20 + m21 * m21 + m22 * m22)
    return centers, cov, lo, hi


def depth_range(mv, lo, hi):
    mv = [float(v) for v in np.asarray(mv, np.float32).reshape(16)]
    near, far = math.inf, -math.inf
    for k in range(8):
        x = hi[0] if k & 1 else lo[0]
        y = hi[1] if k & 2 else lo[1]
        z = hi[2] if k & 4 else lo[2]
        d = -(mv[2] * x + mv[6] * y + mv[10] * z + mv[14])
        near = min(near, d) if d < near else near
        far = d if d > far else far
    if far <= 0:
        return False, F(0), F(0)
    near = max(near, 0.0)
    return True, F(near), F(65535 / max(far - near, 1e-6))


def _clamp(e, lo, hi):
    return np.fmin(np.fmax(e, lo), hi)


def footprint(cov6, view, P, viewport, mv):
    S = [[cov6[0], cov6[1], cov6[2]], [cov6[1], cov6[3], cov6[4]], [cov6[2], cov6[4], cov6[5]]]
    fx = (P[0] * viewport[0]) * F(0.5)
    fy = (P[5] * viewport[1]) * F(0.5)
    z0 = F(0)
    J = [[fx, z0, z0], [z0, fy, z0], [z0, z0, z0]]
    if P[15] == 0:
        d = -view[2]
        x = _clamp(view[0] / d, F(-1.3) / P[0], F(1.3) / P[0]) * d
        y = _clamp(view[1] / d, F(-1.3) / P[5], F(1.3) / P[5]) * d
        J[0][0] = fx / d
        J[1][1] = fy / d
        J[0][2] = (fx * x) / (d * d)
        J[1][2] = (fy * y) / (d * d)
    W = [[mv[c * 4 + r] for c in range(3)] for r in range(3)]
    T = [[(J[r][0] * W[0][c] + J[r][1] * W[1][c]) + J[r][2] * W[2][c] for c in range(3)] for r in range(2)]
    U = [[(T[r][0] * S[0][c] + T[r][1] * S[1][c]) + T[r][2] * S[2][c] for c in range(3)] for r in range(2)]
    fxx = (U[0][0] * T[0][0] + U[0][1] * T[0][1]) + U[0][2] * T[0][2]
    fxy = (U[1][0] * T[0][0] + U[1][1] * T[0][1]) + U[1][2] * T[0][2]
    fyy = (U[1][0] * T[1][0] + U[1][1] * T[1][1]) + U[1][2] * T[1][2]
    return fxx, fxy, fyy


def key(centers, cov, i, mv, P, viewport, depth_min, depth_scale, cull):
    mv = [F(v) for v in np.asarray(mv, np.float32).reshape(16)]
    P = [F(v) for v in np.asarray(P, np.float32).reshape(16)]
    viewport = [F(v) for v in np.asarray(viewport, np.float32).reshape(2)]
    x, y, z = (F(v) for v in centers[i, :3])
    word = int(centers.view(np.uint32)[i, 3])
    view = [((mv[j] * x + mv[4 + j] * y) + mv[8 + j] * z) + mv[12 + j] * F(1) for j in range(4)]
    clip = [((P[j] * view[0] + P[4 + j] * view[1]) + P[8 + j] * view[2]) + P[12 + j] * view[3] for j in range(4)]
    w = clip[3]
    if view[2] >= 0 or clip[2] > w or abs(clip[0]) > F(1.3) * w or abs(clip[1]) > F(1.3) * w:
        return CULLED
    alpha = F(word >> 24) / F(255)
    if alpha * F(255) <= F(1):
        return CULLED
    cull = F(cull)
    if cull > 0:
        fxx, fxy, fyy = footprint([F(v) for v in cov[i]], view, P, viewport, mv)
        det = (fxx + F(0.3)) * (fyy + F(0.3)) - fxy * fxy
        area = F(6.2831853) * np.sqrt(np.fmax(det, F(0)))
        if alpha * area < cull:
            return CULLED
    scaled = (-view[2] - F(depth_min)) * F(depth_scale)
    bucket = int(_clamp(scaled, F(0), F(BUCKETS - 1)))
    return BUCKETS - 1 - bucket


def sort_view(data: bytes, mv, P, viewport, cull):
    """(order, sorted_keys) as lists."""
    centers, cov, lo, hi = decode(data)
    visible, dmin, dscale = depth_range(mv, lo, hi)
    if not visible:
        return [], []
    keys = [key(centers, cov, i, mv, P, viewport, dmin, dscale, cull) for i in range(len(centers))]
    pairs = sorted((k, i) for i, k in enumerate(keys) if k != CULLED)
    return [i for _, i in pairs], [k for k, _ in pairs]
