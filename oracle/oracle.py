"""ctypes front end of the CPU oracle (oracle.cpp).

TEST INFRASTRUCTURE ONLY. Tests, the smoke check and the benchmark's
CPU-baseline leg use this as the checker; the product package never imports
it. See oracle.h for which reference function each entry restates.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
CULLED = 0xFFFFFFFF
BUCKETS = 65536

_lib = None


def build() -> None:
    """Compiles liboracle.so with the Makefile beside this file."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_u8p = ctypes.POINTER(ctypes.c_uint8)


class OrCloud(ctypes.Structure):
    _fields_ = [
        ("model_view", ctypes.c_float * 16),
        ("projection", ctypes.c_float * 16),
        ("viewport", ctypes.c_float * 2),
        ("depth_min", ctypes.c_float),
        ("depth_scale", ctypes.c_float),
        ("count", ctypes.c_uint32),
        ("cull", ctypes.c_float),
    ]


def _declare(L):
    L.or_parse_splat.restype = ctypes.c_int
    L.or_parse_splat.argtypes = [_u8p, ctypes.c_size_t, _f32p, _f32p, _f64p, _f64p, _u32p,
                                 ctypes.c_char_p, ctypes.c_size_t]
    L.or_depth_range.restype = ctypes.c_int
    L.or_depth_range.argtypes = [_f32p, _f64p, _f64p, _f32p, _f32p]
    L.or_key.restype = ctypes.c_uint32
    L.or_key.argtypes = [ctypes.POINTER(OrCloud), _f32p, _f32p, ctypes.c_uint32]
    L.or_footprint.restype = None
    L.or_footprint.argtypes = [ctypes.POINTER(OrCloud), _f32p, ctypes.c_uint32, _f32p, _f32p]
    L.or_make_keys.restype = None
    L.or_make_keys.argtypes = [ctypes.POINTER(OrCloud), _f32p, _f32p, ctypes.c_uint32,
                               ctypes.c_uint32, _u32p]
    L.or_counting_sort.restype = ctypes.c_uint32
    L.or_counting_sort.argtypes = [_u32p, ctypes.c_uint32, _u32p, _u32p]
    L.or_drawlist_sort.restype = None
    L.or_drawlist_sort.argtypes = [_u32p, _u32p, ctypes.c_uint32, _u32p, _u32p]
    L.or_shade.restype = ctypes.c_uint32
    L.or_shade.argtypes = [_f32p, _u32p, ctypes.c_int, ctypes.c_uint32, _f32p]
    L.or_particle_key.restype = ctypes.c_uint32
    L.or_particle_key.argtypes = [_f32p, _f32p, _f32p]
    L.or_particle_sort.restype = ctypes.c_uint32
    L.or_particle_sort.argtypes = [_f32p, ctypes.c_uint32, ctypes.c_uint32, _f32p, _f32p, _u32p, _u32p]
    L.or_sort_view.restype = ctypes.c_uint32
    L.or_sort_view.argtypes = [_f32p, _f32p, ctypes.c_uint32, _f64p, _f64p, _f32p, _f32p, _f32p,
                               ctypes.c_float, _u32p, _u32p, ctypes.c_int]


def _ptr(a: np.ndarray, t):
    return a.ctypes.data_as(t)


class OracleError(ValueError):
    def __init__(self, code: int, message: str, bad_index: int | None = None):
        super().__init__(message)
        self.code = code
        self.bad_index = bad_index


class Parsed:
    """What parseSplatFile returns: count, centers (4 f32 a splat, the 4th the
    colour word's bits), covariances (6 f32 a splat), min, max (doubles)."""

    def __init__(self, count, centers, covariances, bmin, bmax):
        self.count = count
        self.centers = centers
        self.covariances = covariances
        self.min = bmin
        self.max = bmax

    @property
    def colours(self) -> np.ndarray:
        return self.centers.view(np.uint32)[:, 3]


def parse_splat(data: bytes | np.ndarray) -> Parsed:
    buf = np.frombuffer(bytes(data), dtype=np.uint8) if not isinstance(data, np.ndarray) else data
    buf = np.ascontiguousarray(buf, dtype=np.uint8)
    n = buf.size // 32 if buf.size % 32 == 0 else 0
    centers = np.zeros((max(n, 1), 4), np.float32)
    cov = np.zeros((max(n, 1), 6), np.float32)
    bmin = np.zeros(3, np.float64)
    bmax = np.zeros(3, np.float64)
    bad = np.zeros(1, np.uint32)
    err = ctypes.create_string_buffer(256)
    rc = lib().or_parse_splat(_ptr(buf, _u8p), buf.size, _ptr(centers, _f32p), _ptr(cov, _f32p),
                              _ptr(bmin, _f64p), _ptr(bmax, _f64p), _ptr(bad, _u32p), err, 256)
    if rc != 0:
        raise OracleError(rc, err.value.decode(), int(bad[0]) if rc == -4 else None)
    return Parsed(n, centers[:n], cov[:n], bmin, bmax)


def depth_range(model_view, bmin, bmax):
    """(visible, depth_min, depth_scale) as the reference's prepare computes them."""
    mv = np.ascontiguousarray(model_view, np.float32).reshape(16)
    lo = np.ascontiguousarray(bmin, np.float64)
    hi = np.ascontiguousarray(bmax, np.float64)
    dmin = np.zeros(1, np.float32)
    dscale = np.zeros(1, np.float32)
    rc = lib().or_depth_range(_ptr(mv, _f32p), _ptr(lo, _f64p), _ptr(hi, _f64p), _ptr(dmin, _f32p),
                              _ptr(dscale, _f32p))
    return rc == 0, dmin[0], dscale[0]


def make_cloud(model_view, projection, viewport, depth_min, depth_scale, count, cull) -> OrCloud:
    c = OrCloud()
    c.model_view[:] = [float(v) for v in np.asarray(model_view, np.float32).reshape(16)]
    c.projection[:] = [float(v) for v in np.asarray(projection, np.float32).reshape(16)]
    c.viewport[:] = [float(v) for v in np.asarray(viewport, np.float32).reshape(2)]
    c.depth_min = float(depth_min)
    c.depth_scale = float(depth_scale)
    c.count = int(count)
    c.cull = float(cull)
    return c


def make_keys(parsed: Parsed, model_view, projection, viewport, cull) -> np.ndarray:
    """Per-splat keys (CULLED for culled splats), or all CULLED when the
    cloud is wholly behind the camera."""
    n = parsed.count
    visible, dmin, dscale = depth_range(model_view, parsed.min, parsed.max)
    keys = np.full(n, CULLED, np.uint32)
    if not visible:
        return keys
    c = make_cloud(model_view, projection, viewport, dmin, dscale, n, cull)
    lib().or_make_keys(ctypes.byref(c), _ptr(parsed.centers, _f32p), _ptr(parsed.covariances, _f32p),
                       0, n, _ptr(keys, _u32p))
    return keys


def counting_sort(keys: np.ndarray):
    keys = np.ascontiguousarray(keys, np.uint32)
    n = keys.size
    order = np.zeros(max(n, 1), np.uint32)
    sk = np.zeros(max(n, 1), np.uint32)
    s = lib().or_counting_sort(_ptr(keys, _u32p), n, _ptr(order, _u32p), _ptr(sk, _u32p))
    return order[:s].copy(), sk[:s].copy()


def drawlist_sort(keys, payloads):
    k = np.array(keys, dtype=np.uint32)
    p = np.array(payloads, dtype=np.uint32)
    n = k.size
    ka = np.zeros(max(n, 1), np.uint32)
    pa = np.zeros(max(n, 1), np.uint32)
    if n:
        lib().or_drawlist_sort(_ptr(k, _u32p), _ptr(p, _u32p), n, _ptr(ka, _u32p), _ptr(pa, _u32p))
    return k, p


def sort_view(parsed: Parsed, model_view, projection, viewport, cull, threads: int = 1):
    """(order, sorted_keys) for one view: range, keys and the stable sort."""
    n = parsed.count
    order = np.zeros(max(n, 1), np.uint32)
    sk = np.zeros(max(n, 1), np.uint32)
    mv = np.ascontiguousarray(model_view, np.float32).reshape(16)
    pr = np.ascontiguousarray(projection, np.float32).reshape(16)
    vp = np.ascontiguousarray(viewport, np.float32).reshape(2)
    s = lib().or_sort_view(_ptr(parsed.centers, _f32p), _ptr(parsed.covariances, _f32p), n,
                           _ptr(parsed.min, _f64p), _ptr(parsed.max, _f64p), _ptr(mv, _f32p),
                           _ptr(pr, _f32p), _ptr(vp, _f32p), float(np.float32(cull)),
                           _ptr(order, _u32p), _ptr(sk, _u32p), int(threads))
    return order[:s].copy(), sk[:s].copy()


PARTICLE_BUCKETS = 4096


def particle_key(particle, eye, forward) -> int:
    """One particle's key (8 f32), or CULLED for a dead slot."""
    p = np.ascontiguousarray(particle, np.float32).reshape(8)
    e = np.ascontiguousarray(eye, np.float32).reshape(3)
    f = np.ascontiguousarray(forward, np.float32).reshape(3)
    return int(lib().or_particle_key(_ptr(p, _f32p), _ptr(e, _f32p), _ptr(f, _f32p)))


def particle_sort(pool: np.ndarray, offset: int, capacity: int, eye, forward):
    """(order, sorted_keys) of one emitter: the live slots by (key, slot)."""
    pool = np.ascontiguousarray(pool, np.float32).reshape(-1)
    if pool.size < 8 * (offset + capacity):
        raise ValueError("the pool is shorter than the ring")
    order = np.zeros(max(capacity, 1), np.uint32)
    sk = np.zeros(max(capacity, 1), np.uint32)
    e = np.ascontiguousarray(eye, np.float32).reshape(3)
    f = np.ascontiguousarray(forward, np.float32).reshape(3)
    s = lib().or_particle_sort(_ptr(pool, _f32p), offset, capacity, _ptr(e, _f32p), _ptr(f, _f32p),
                               _ptr(order, _u32p), _ptr(sk, _u32p))
    return order[:s].copy(), sk[:s].copy()


def shade(centers: np.ndarray, sh: np.ndarray, degree: int, indices, eye) -> np.ndarray:
    """The shade pass's colour word for each splat index given."""
    c = np.ascontiguousarray(centers, np.float32).reshape(-1)
    w = np.ascontiguousarray(sh, np.uint32).reshape(-1)
    e = np.ascontiguousarray(eye, np.float32).reshape(3)
    L = lib()
    cp, wp, ep = _ptr(c, _f32p), _ptr(w, _u32p), _ptr(e, _f32p)
    return np.array([L.or_shade(cp, wp, degree, int(i), ep) for i in indices], np.uint32)
