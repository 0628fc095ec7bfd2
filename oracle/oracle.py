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
    L.or_exp.restype = ctypes.c_double
    L.or_exp.argtypes = [ctypes.c_double]
    L.or_byte.restype = ctypes.c_uint32
    L.or_byte.argtypes = [ctypes.c_double]
    L.or_signed_half.restype = ctypes.c_uint32
    L.or_signed_half.argtypes = [ctypes.c_double]
    L.or_decode_ply.restype = ctypes.c_int
    L.or_decode_ply.argtypes = [_u8p, ctypes.c_uint32, ctypes.c_uint32, _u32p, _u32p, ctypes.c_uint32, _f32p,
                                _f32p, _u32p, _f64p, _f64p, _u32p]
    L.or_decode_spz.restype = ctypes.c_int
    L.or_decode_spz.argtypes = [_u8p, ctypes.c_size_t, _u32p, _u32p, _f32p, _f32p, _u32p, _f64p, _f64p, _u32p,
                                ctypes.c_char_p, ctypes.c_size_t]
    L.or_decode_sog.restype = ctypes.c_int
    L.or_decode_sog.argtypes = [ctypes.c_uint32, ctypes.c_uint32] + [_u8p] * 7 + [
        ctypes.c_uint32, ctypes.c_size_t, _f64p, _f64p, _f64p, _f64p, _f64p, ctypes.c_double, _f32p, _f32p, _u32p,
        _f64p, _f64p, _u32p]
    L.or_draw_tables.restype = None
    L.or_draw_tables.argtypes = [_f32p, _f32p]
    L.or_draw.restype = None
    L.or_draw.argtypes = [_f32p, _f32p, _u32p, ctypes.c_uint32, _u32p, _f32p, _f32p, ctypes.c_uint32,
                          ctypes.c_uint32, _f32p]
    L.or_draw_cut_check.restype = None
    L.or_draw_cut_check.argtypes = [_f32p, _f32p, _u32p, ctypes.c_uint32, _f32p, _f32p, ctypes.c_uint32,
                                    ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint64)]
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


# ------------------------------------------------------------ capture readers

SH_COEFFICIENTS = (0, 3, 8, 15)
PLY_TYPES = {   # scene/splats.js:391-396: name -> (type code, bytes)
    "char": (1, 1), "int8": (1, 1), "uchar": (2, 1), "uint8": (2, 1),
    "short": (3, 2), "int16": (3, 2), "ushort": (4, 2), "uint16": (4, 2),
    "int": (5, 4), "int32": (5, 4), "uint": (6, 4), "uint32": (6, 4),
    "float": (7, 4), "float32": (7, 4), "double": (8, 8), "float64": (8, 8),
}
PLY_NEEDS = ["x", "y", "z", "f_dc_0", "f_dc_1", "f_dc_2", "opacity", "scale_0", "scale_1", "scale_2",
             "rot_0", "rot_1", "rot_2", "rot_3"]


def sh_words(degree: int) -> int:
    return (SH_COEFFICIENTS[degree] * 3 + 1) // 2


class Capture(Parsed):
    """A decoded capture with its harmonics: degree and sh (uint32 words)."""

    def __init__(self, count, centers, covariances, bmin, bmax, degree=0, sh=None):
        super().__init__(count, centers, covariances, bmin, bmax)
        self.degree = degree
        self.sh = sh if sh is not None else np.zeros(1, np.uint32)


def _js_number_text(v: float) -> str:
    if v != v:
        return "NaN"
    if v == int(v) and abs(v) < 1e21:
        return str(int(v))
    return repr(v)


def _to_number(word):
    if word is None:
        return float("nan")
    t = word.strip()
    if t == "":
        return 0.0
    try:
        if t[:2].lower() in ("0x", "0o", "0b"):
            return float(int(t, 0))
        if t in ("Infinity", "+Infinity", "-Infinity"):
            return float(t.replace("Infinity", "inf"))
        if any(ch not in "0123456789+-.eE" for ch in t):
            return float("nan")
        return float(t)
    except ValueError:
        return float("nan")


def parse_ply(data: bytes) -> Capture:
    """parsePly (scene/splats.js:398-468): the header restated here, the
    per-vertex arithmetic in oracle.cpp."""
    data = bytes(data)
    marker = b"end_header"
    end = -1
    for i in range(min(len(data), 65536) - len(marker)):
        if data[i:i + len(marker)] == marker:
            end = i + len(marker)
            break
    if end < 0:
        raise OracleError(-5, "splats: a .ply with no end_header")
    if end < len(data) and data[end] == 0x0D:
        end += 1
    end += 1
    header = data[:end].decode("utf-8", "replace").replace("\r\n", "\n").split("\n")
    fmt = "null"
    vertices = None
    for line in header:
        words = line.strip().split() or [""]
        w = lambda k: words[k] if k < len(words) else None
        if words[0] == "format":
            fmt = w(1) if w(1) is not None else "undefined"
        elif words[0] == "element":
            kind = w(1) if w(1) is not None else "undefined"
            if vertices is None and kind == "chunk":
                raise OracleError(-5, "splats: a compressed .ply (from SuperSplat) is not read; export an "
                                      "uncompressed .ply or a .splat")
            if vertices is None and kind != "vertex":
                raise OracleError(-5, f"splats: a .ply whose first element is '{kind}', not 'vertex'")
            if vertices is not None:
                break
            vertices = {"count": _to_number(w(2)), "props": {}, "stride": 0}
        elif words[0] == "property" and vertices is not None:
            t = w(1) if w(1) is not None else "undefined"
            if t == "list":
                raise OracleError(-5, "splats: a .ply with list properties on its vertices is not a splat capture")
            if t not in PLY_TYPES:
                raise OracleError(-5, f"splats: unknown .ply property type '{t}'")
            name = w(2) if w(2) is not None else "undefined"
            vertices["props"][name] = (PLY_TYPES[t][0], vertices["stride"])
            vertices["stride"] += PLY_TYPES[t][1]
    if vertices is None:
        raise OracleError(-5, "splats: a .ply with no vertices")
    if fmt != "binary_little_endian":
        raise OracleError(-5, f"splats: a .ply in '{fmt}' format; only binary_little_endian is read")
    count = vertices["count"]
    if not (count == count and count != float("inf") and count == int(count) and count > 0):
        raise OracleError(-5, f"splats: a .ply with {_js_number_text(count)} vertices")
    props = vertices["props"]
    missing = [n for n in PLY_NEEDS if n not in props]
    if missing:
        raise OracleError(-5, f"splats: this .ply is not a splat capture: no {', '.join(missing)}")
    stride = vertices["stride"]
    n = int(count)
    if end + n * stride > len(data):
        raise OracleError(-5, f"splats: the .ply is cut short: {n} vertices need {n * stride} bytes, "
                              f"it has {len(data) - end}")
    rest = 0
    while f"f_rest_{rest}" in props:
        rest += 1
    degree = SH_COEFFICIENTS.index(rest // 3) if rest % 3 == 0 and rest // 3 in SH_COEFFICIENTS else -1
    if rest > 0 and degree < 1:
        raise OracleError(-5, f"splats: a .ply with {rest} f_rest_ properties; harmonics of degree 1, 2 or 3 "
                              "have 9, 24 or 45")
    degree = max(degree, 0)
    names = PLY_NEEDS + [f"f_rest_{k}" for k in range(rest)]
    types = np.array([props[nm][0] for nm in names], np.uint32)
    offsets = np.array([props[nm][1] for nm in names], np.uint32)
    payload = np.frombuffer(data, np.uint8, count=n * stride, offset=end).copy()
    centers = np.zeros((n, 4), np.float32)
    cov = np.zeros((n, 6), np.float32)
    sh = np.zeros(n * sh_words(degree) + 1 if degree else 1, np.uint32)
    bmin = np.zeros(3, np.float64)
    bmax = np.zeros(3, np.float64)
    bad = ctypes.c_uint32(0)
    rc = lib().or_decode_ply(_ptr(payload, _u8p), n, stride, _ptr(types, _u32p), _ptr(offsets, _u32p), rest,
                             _ptr(centers, _f32p), _ptr(cov, _f32p), _ptr(sh, _u32p), _ptr(bmin, _f64p),
                             _ptr(bmax, _f64p), ctypes.byref(bad))
    if rc == -4:
        raise OracleError(-4, f"splats: splat {bad.value} has a position that is not a number", bad.value)
    return Capture(n, centers, cov, bmin, bmax, degree, sh)


def parse_spz(gz: bytes) -> Capture:
    """parseSpz (scene/splats.js:227-303) after gunzip (the reference's
    DecompressionStream)."""
    import zlib
    data = np.frombuffer(zlib.decompress(bytes(gz), 16 + zlib.MAX_WBITS), np.uint8).copy()
    count = ctypes.c_uint32(0)
    degree = ctypes.c_uint32(0)
    err = ctypes.create_string_buffer(256)
    bad = ctypes.c_uint32(0)
    z3 = np.zeros(3, np.float64)
    L = lib()
    rc = L.or_decode_spz(_ptr(data, _u8p), data.size, ctypes.byref(count), ctypes.byref(degree), None, None, None,
                         _ptr(z3, _f64p), _ptr(z3, _f64p), ctypes.byref(bad), err, 256)
    if rc:
        raise OracleError(rc, err.value.decode())
    n, d = count.value, degree.value
    centers = np.zeros((n, 4), np.float32)
    cov = np.zeros((n, 6), np.float32)
    sh = np.zeros(n * sh_words(d) + 1 if d else 1, np.uint32)
    bmin = np.zeros(3, np.float64)
    bmax = np.zeros(3, np.float64)
    rc = L.or_decode_spz(_ptr(data, _u8p), data.size, ctypes.byref(count), ctypes.byref(degree), _ptr(centers, _f32p),
                         _ptr(cov, _f32p), _ptr(sh, _u32p), _ptr(bmin, _f64p), _ptr(bmax, _f64p), ctypes.byref(bad),
                         err, 256)
    if rc == -4:
        raise OracleError(-4, f"splats: splat {bad.value} has a position that is not a number", bad.value)
    return Capture(n, centers, cov, bmin, bmax, d, sh)


# ------------------------------------------------------------------ .sog

class _Undefined:
    """JavaScript's undefined: a property the parsed meta.json does not have."""

    def __repr__(self):
        return "undefined"


UNDEFINED = _Undefined()


def js_string(v) -> str:
    """String(v) for a value JSON.parse can give (or undefined)."""
    if v is UNDEFINED:
        return "undefined"
    if v is None:
        return "null"
    if v is True or v is False:
        return "true" if v else "false"
    if isinstance(v, (int, float)):
        return js_number_string(float(v))
    if isinstance(v, str):
        return v
    if isinstance(v, list):   # Array.prototype.join: null and undefined as ""
        return ",".join("" if (x is None or x is UNDEFINED) else js_string(x) for x in v)
    return "[object Object]"


def js_number_string(v: float) -> str:
    """Number::toString (ECMA-262 6.1.6.1.20) from the shortest round-trip digits."""
    if v != v:
        return "NaN"
    if v == 0:
        return "0"
    if v in (float("inf"), float("-inf")):
        return "Infinity" if v > 0 else "-Infinity"
    if v < 0:
        return "-" + js_number_string(-v)
    mant, _, exp = repr(v).partition("e")
    ip, _, fp = mant.partition(".")
    digits = (ip + fp).lstrip("0")
    lead = len(ip + fp) - len((ip + fp).lstrip("0"))
    n = len(ip) - lead + (int(exp) if exp else 0)   # value = 0.digits x 10^n
    digits = digits.rstrip("0")
    k = len(digits)
    if k <= n <= 21:
        return digits + "0" * (n - k)
    if 0 < n <= 21:
        return digits[:n] + "." + digits[n:]
    if -6 < n <= 0:
        return "0." + "0" * (-n) + digits
    e = n - 1
    return digits[0] + ("." + digits[1:] if k > 1 else "") + "e" + ("+" if e >= 0 else "-") + str(abs(e))


def js_to_number(v) -> float:
    """ToNumber(v) for a value JSON.parse can give (or undefined)."""
    if v is UNDEFINED:
        return float("nan")
    if v is None or v is False:
        return 0.0
    if v is True:
        return 1.0
    if isinstance(v, (int, float)):
        return float(v)
    if isinstance(v, str):
        return _to_number(v)
    return _to_number(js_string(v))   # ToPrimitive of an array or object is its string


def _get(v, key):
    """v[key] in JavaScript for JSON values; None when that would throw (v
    null or undefined)."""
    if v is None or v is UNDEFINED:
        return None
    if isinstance(v, dict):
        return v.get(str(key), UNDEFINED)
    if isinstance(v, list):
        return v[key] if isinstance(key, int) and 0 <= key < len(v) else UNDEFINED
    if isinstance(v, str):
        return v[key] if isinstance(key, int) and 0 <= key < len(v) else UNDEFINED
    return UNDEFINED


def _truthy(v) -> bool:
    if v is None or v is UNDEFINED or v is False:
        return False
    if isinstance(v, (int, float)) and not isinstance(v, bool):
        return not (v == 0 or v != v)
    if isinstance(v, str):
        return v != ""
    return True


def _unzip(data: bytes) -> dict:
    """The zip directory walk of readSplats (scene/splats.js:95-125): name ->
    entry bytes (deflated entries inflated), stored and deflate only."""
    import zlib
    n = len(data)
    u16 = lambda o: int.from_bytes(data[o:o + 2], "little")
    u32 = lambda o: int.from_bytes(data[o:o + 4], "little")
    end = -1
    for i in range(n - 22, max(0, n - 22 - 65535) - 1, -1):
        if i >= 0 and u32(i) == 0x06054B50:
            end = i
            break
    if end < 0:
        raise OracleError(-20, "splats: a zip with no end record: cut short?")
    files = {}
    at = u32(end + 16)
    for _ in range(u16(end + 10)):
        if at + 46 > n or u32(at) != 0x02014B50:
            raise OracleError(-21, "splats: a zip whose directory is damaged")
        method, size, name_len, local = u16(at + 10), u32(at + 20), u16(at + 28), u32(at + 42)
        name = data[at + 46:at + 46 + name_len].decode("utf-8", "replace")
        if name.startswith("\ufeff"):
            name = name[1:]
        if size == 0xFFFFFFFF or local == 0xFFFFFFFF:
            raise OracleError(-22, "splats: a zip64 .sog is not read")
        at += 46 + name_len + u16(at + 30) + u16(at + 32)
        start = local + 30 + u16(local + 26) + u16(local + 28)
        if start + size > n:
            raise OracleError(-23, f"splats: the zip is cut short in {name}")
        stored = data[start:start + size]
        if method not in (0, 8):
            raise OracleError(-24, f"splats: {name} is compressed with method {method}; stored and deflate are read")
        files[name] = (method, stored)
    return files


def _inflate(entry) -> bytes:
    import zlib
    method, stored = entry
    return bytes(stored) if method == 0 else zlib.decompress(bytes(stored), -15)


def parse_sog(data: bytes, decode_image=None) -> Capture:
    """readSog (scene/splats.js:127-200): the container, meta.json and the
    checks restated here with the reference's messages, in its order; the
    per-splat loop in oracle.cpp. decode_image(bytes) -> (width, height,
    rgba) plays the reference's decodeImage."""
    import json
    if decode_image is None:
        raise OracleError(-25, "splats: a .sog needs decodeImage, for its WebP images")
    data = bytes(data)
    files = _unzip(data)

    def file(name):
        if not isinstance(name, str) or name not in files:
            raise OracleError(-26, f"splats: the .sog has no {js_string(name)}")
        return _inflate(files[name])

    text = file("meta.json").decode("utf-8", "replace")
    if text.startswith("\ufeff"):
        text = text[1:]
    try:
        meta = json.loads(text)
    except ValueError:
        raise OracleError(-27, "splats: the .sog's meta.json is not JSON")
    version = _get(meta, "version")
    if version is None:
        raise OracleError(-28, "splats: the .sog's meta.json has no version")
    if not (isinstance(version, (int, float)) and not isinstance(version, bool) and version == 2):
        shown = "1" if version is UNDEFINED or version is None else js_string(version)
        raise OracleError(-29, f"splats: a .sog of version {shown}; version 2 is read (re-save it with splat-transform)")
    count = _get(meta, "count")
    if not (isinstance(count, (int, float)) and not isinstance(count, bool) and count == count
            and float(count).is_integer() and count > 0):
        raise OracleError(-30, f"splats: a .sog of {js_string(count)} splats")
    count = int(count)

    def member(path):
        """meta.path; reading a property of null or undefined (JavaScript's
        TypeError) names the member that is missing."""
        v, shown = meta, []
        for key in path:
            if v is None or v is UNDEFINED:
                raise OracleError(-31, "splats: the .sog's meta.json has no " + ".".join(shown))
            v = _get(v, key)
            shown.append(str(key))
        return v

    def decoded(name):
        w, h, rgba = decode_image(file(name))
        return int(w), int(h), np.frombuffer(bytes(rgba), np.uint8)

    names = [member(("means", "files", 0)), member(("means", "files", 1)), member(("quats", "files", 0)),
             member(("scales", "files", 0)), member(("sh0", "files", 0))]
    for nm in names:
        file(nm)
    images = []
    for nm in names:
        w, h, rgba = decoded(nm)
        if w * h < count:
            raise OracleError(-32, f"splats: {js_string(nm)} has {w * h} pixels, for {count} splats")
        images.append(rgba)
    shn = _get(meta, "shN")
    bands = _get(shn, "bands") if _truthy(shn) else 0
    if bands is None:
        bands = UNDEFINED
    key = js_string(bands) if isinstance(bands, str) else (js_number_string(float(bands))
                                                              if isinstance(bands, (int, float)) and not isinstance(bands, bool) else None)
    degree = int(key) if key in ("1", "2", "3") else 0
    per = SH_COEFFICIENTS[degree]
    labels = np.zeros(4, np.uint8)
    palette = np.zeros(4, np.uint8)
    pw = 0
    if degree > 0:
        pw, _, palette = decoded(member(("shN", "files", 0)))
        lname = member(("shN", "files", 1))
        lw, lh, labels = decoded(lname)
        if lw * lh < count:
            raise OracleError(-32, f"splats: {js_string(lname)} has {lw * lh} pixels, for {count} splats")
        if pw != 64 * per:
            raise OracleError(-33, f"splats: the .sog's harmonic palette is {pw} wide; {64 * per} for degree {degree}")

    def book(path):
        b = member(path)
        if b is None or b is UNDEFINED:
            raise OracleError(-31, "splats: the .sog's meta.json has no " + ".".join(path))
        return np.array([js_to_number(_get(b, k)) for k in range(256)], np.float64)

    def triple(path):
        b = member(path)
        if b is None or b is UNDEFINED:
            raise OracleError(-31, "splats: the .sog's meta.json has no " + ".".join(path))
        return np.array([js_to_number(_get(b, k)) for k in range(3)], np.float64)

    mins, maxs = triple(("means", "mins")), triple(("means", "maxs"))
    colour_book = book(("sh0", "codebook"))
    scale_book = book(("scales", "codebook"))
    sh_book = book(("shN", "codebook")) if degree > 0 else np.zeros(256, np.float64)
    sh_count = js_to_number(_get(shn, "count")) if degree > 0 else 0.0
    pix = [np.ascontiguousarray(im[:count * 4]) for im in images]
    lab = np.ascontiguousarray(labels[:count * 4]) if degree > 0 else np.zeros(4, np.uint8)
    pal = np.ascontiguousarray(palette)
    centers = np.zeros((count, 4), np.float32)
    cov = np.zeros((count, 6), np.float32)
    sh = np.zeros(count * sh_words(degree) + 1 if degree else 1, np.uint32)
    bmin = np.zeros(3, np.float64)
    bmax = np.zeros(3, np.float64)
    bad = ctypes.c_uint32(0)
    rc = lib().or_decode_sog(count, degree, *[_ptr(p, _u8p) for p in pix], _ptr(lab, _u8p), _ptr(pal, _u8p), pw,
                             pal.size, _ptr(mins, _f64p), _ptr(maxs, _f64p), _ptr(scale_book, _f64p),
                             _ptr(colour_book, _f64p), _ptr(sh_book, _f64p), sh_count, _ptr(centers, _f32p),
                             _ptr(cov, _f32p), _ptr(sh, _u32p), _ptr(bmin, _f64p), _ptr(bmax, _f64p),
                             ctypes.byref(bad))
    if rc == -4:
        raise OracleError(-4, f"splats: splat {bad.value} has a position that is not a number", bad.value)
    return Capture(count, centers, cov, bmin, bmax, degree, sh)


def draw_tables():
    srgb = np.zeros(256, np.float32)
    reach = np.zeros(256, np.float32)
    lib().or_draw_tables(_ptr(srgb, _f32p), _ptr(reach, _f32p))
    return srgb, reach


def draw_cut_check(parsed, order, model_view, projection, width: int, height: int):
    """(covered pixels the draw's box cut would leave out, covered pixels,
    pinned box pixels, cut box pixels) over the splats of order
    (or_draw_cut_check)."""
    out = np.zeros(4, np.uint64)
    o = np.ascontiguousarray(order, np.uint32)
    mv = np.ascontiguousarray(model_view, np.float32).reshape(16)
    pr = np.ascontiguousarray(projection, np.float32).reshape(16)
    lib().or_draw_cut_check(_ptr(parsed.centers, _f32p), _ptr(parsed.covariances, _f32p), _ptr(o, _u32p), o.size,
                            _ptr(mv, _f32p), _ptr(pr, _f32p), width, height,
                            out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)))
    return tuple(int(v) for v in out)


def draw(parsed, order, model_view, projection, width: int, height: int, background=None, shaded=None):
    """The pinned splat draw: an RGBA f32 image (height, width, 4)."""
    img = np.zeros((height, width, 4), np.float32) if background is None else \
        np.array(background, np.float32).reshape(height, width, 4).copy()
    o = np.ascontiguousarray(order, np.uint32)
    sh = None if shaded is None else np.ascontiguousarray(shaded, np.uint32)
    mv = np.ascontiguousarray(model_view, np.float32).reshape(16)
    pr = np.ascontiguousarray(projection, np.float32).reshape(16)
    lib().or_draw(_ptr(parsed.centers, _f32p), _ptr(parsed.covariances, _f32p), _ptr(o, _u32p), o.size,
                  None if sh is None else _ptr(sh, _u32p), _ptr(mv, _f32p), _ptr(pr, _f32p), width, height,
                  _ptr(img, _f32p))
    return img
