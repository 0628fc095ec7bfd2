"""Camera matrices as the reference builds them: FP64 arithmetic, stored f32.

These produce the f32 view and projection a caller hands to the sort (the
values the reference writes into its Cloud uniform). Restated from, in the
reference project:
  mat4Multiply                     src/core/math/mat4.js:96-130
  mat4LookAt                       src/core/math/mat4.js:243-275
  mat4PerspectiveReverseZInfinite  src/core/math/mat4.js:455-468
  fitDistance / boundsRadius       src/scene/camera.js:45-62
  Camera.update                    src/scene/camera.js:258-276
All matrices are column-major float32[16], as WGSL and the reference store them.
"""
from __future__ import annotations

import math

import numpy as np


def _f32(v) -> list[float]:
    return [float(x) for x in np.asarray(v, np.float32).reshape(-1)]


def hypot3(x: float, y: float, z: float) -> float:
    return math.sqrt(x * x + y * y + z * z)


def mat4_multiply(a, b) -> np.ndarray:
    """out = a * b, products and sums in doubles, stored as float32."""
    a = _f32(a)
    b = _f32(b)
    out = np.zeros(16, np.float32)
    for col in range(4):
        b0, b1, b2, b3 = b[col * 4:col * 4 + 4]
        for row in range(4):
            out[col * 4 + row] = b0 * a[row] + b1 * a[4 + row] + b2 * a[8 + row] + b3 * a[12 + row]
    return out


def look_at(eye, center, up=(0.0, 1.0, 0.0)) -> np.ndarray:
    eye = _f32(eye)
    center = _f32(center)
    up = _f32(up)
    zx, zy, zz = eye[0] - center[0], eye[1] - center[1], eye[2] - center[2]
    zl = hypot3(zx, zy, zz)
    if not zl > 1e-6:
        raise ValueError("mat4LookAt: eye and center coincide")
    zx /= zl
    zy /= zl
    zz /= zl
    xx = up[1] * zz - up[2] * zy
    xy = up[2] * zx - up[0] * zz
    xz = up[0] * zy - up[1] * zx
    xl = hypot3(xx, xy, xz)
    if not xl > 1e-6:
        raise ValueError("mat4LookAt: up is parallel to the view direction")
    xx /= xl
    xy /= xl
    xz /= xl
    yx = zy * xz - zz * xy
    yy = zz * xx - zx * xz
    yz = zx * xy - zy * xx
    return np.array([
        xx, yx, zx, 0,
        xy, yy, zy, 0,
        xz, yz, zz, 0,
        -(xx * eye[0] + xy * eye[1] + xz * eye[2]),
        -(yx * eye[0] + yy * eye[1] + yz * eye[2]),
        -(zx * eye[0] + zy * eye[1] + zz * eye[2]),
        1,
    ], np.float32)


def perspective(fov_y: float, aspect: float, near: float) -> np.ndarray:
    """Reverse-Z, infinite far: clip z = near, clip w = -view z."""
    if not (0 < fov_y < math.pi and aspect > 0 and near > 0):
        raise ValueError("perspective: fovY in (0, pi), aspect and near positive")
    f = 1 / math.tan(fov_y * 0.5)
    return np.array([f / aspect, 0, 0, 0, 0, f, 0, 0, 0, 0, 0, -1, 0, 0, near, 0], np.float32)


def bounds_radius(lo, hi) -> float:
    return 0.5 * hypot3(hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2])


def fit_distance(radius: float, fov_y: float, aspect: float = 1.0, margin: float = 1.0,
                 near: float = 0.0) -> float:
    if not radius > 0:
        return 0.0
    half_y = fov_y * 0.5
    half_x = math.atan(math.tan(half_y) * (aspect if aspect > 0 else 1))
    fit = (radius / math.sin(min(half_y, half_x))) * margin
    return max(fit, radius + near)


class Camera:
    """The reference Camera's perspective form: position, target, up, fovY, near."""

    def __init__(self, fov_y: float = math.pi / 3, near: float = 0.1):
        self.fov_y = fov_y
        self.near = near
        self.position = np.array([0, 0, 5], np.float32)
        self.target = np.zeros(3, np.float32)
        self.up = np.array([0, 1, 0], np.float32)
        self.view = np.eye(4, dtype=np.float32).reshape(16)
        self.projection = np.eye(4, dtype=np.float32).reshape(16)

    def update(self, aspect: float) -> "Camera":
        self.view = look_at(self.position, self.target, self.up)
        self.projection = perspective(self.fov_y, aspect, self.near)
        return self
