"""Capture formats decoded on the device: .ply and .spz (readSplats,
src/scene/splats.js:78-90, parsePly :398-468, parseSpz :227-303).

CPU: the oracle against the reference's own .ply cases
(test/splats.test.js:73-117) and its refusals (:331-347), the pinned
Math.exp against a 60-digit decimal exponential, and hand-built .spz splats.
GPU: ws_cloud_load against the oracle, bit for bit -- centres, colour words,
covariances, box and harmonics -- over random .ply files (float and mixed
property types, degrees 0-3, extreme opacities and scales) and random .spz
files (versions 1-3, file degrees 0-4), the refusals with the reference's
messages, and a sort of a loaded .ply against the oracle's sort.
"""
import decimal
import gzip
import math
import struct

import numpy as np
import pytest

from oracle import oracle as O

SH_C0 = 0.28209479177387814
PLY_BASE = ["x", "y", "z", "f_dc_0", "f_dc_1", "f_dc_2", "opacity", "scale_0", "scale_1", "scale_2",
            "rot_0", "rot_1", "rot_2", "rot_3"]
FMT = {"char": "b", "uchar": "B", "short": "h", "ushort": "H", "int": "i", "uint": "I", "float": "f",
       "double": "d", "int8": "b", "uint8": "B", "float32": "f", "float64": "d"}


def ply(props, rows, fmt="binary_little_endian", extra_header=""):
    """A .ply of the given (type, name) properties; rows: dicts (missing: 0)."""
    head = (f"ply\nformat {fmt} 1.0\n{extra_header}element vertex {len(rows)}\n"
            + "".join(f"property {t} {n}\n" for t, n in props) + "end_header\n").encode()
    pack = "<" + "".join(FMT[t] for t, _ in props)
    body = b"".join(struct.pack(pack, *[r.get(n, 0) for _, n in props]) for r in rows)
    return head + body


def float_props(names):
    return [("float", n) for n in names]


def random_ply(n, degree, seed, types=None, extremes=False):
    rng = np.random.default_rng(seed)
    rest = [f"f_rest_{k}" for k in range(O.SH_COEFFICIENTS[degree] * 3)]
    names = PLY_BASE[:3] + ["nx", "ny", "nz"] + PLY_BASE[3:] + rest
    props = [((types or {}).get(nm, "float"), nm) for nm in names]
    cols = {
        "x": rng.normal(0, 10, n), "y": rng.normal(0, 10, n), "z": rng.normal(0, 10, n),
        "f_dc_0": rng.normal(0, 1.5, n), "f_dc_1": rng.normal(0, 1.5, n), "f_dc_2": rng.normal(0, 1.5, n),
        "opacity": rng.normal(0, 4, n),
        "scale_0": rng.normal(-4, 1, n), "scale_1": rng.normal(-4, 1, n), "scale_2": rng.normal(-4, 1, n),
        "rot_0": rng.normal(size=n), "rot_1": rng.normal(size=n), "rot_2": rng.normal(size=n),
        "rot_3": rng.normal(size=n),
    }
    for r in rest:
        cols[r] = rng.normal(0, 0.3, n)
    if extremes:
        k = n // 10
        cols["opacity"][:k] = rng.choice([-900.0, 900.0, 37.0, -37.0, 0.0], size=k)
        cols["scale_0"][k:2 * k] = rng.choice([800.0, -800.0, 20.0, -30.0], size=k)
        for q in ("rot_0", "rot_1", "rot_2", "rot_3"):
            cols[q][2 * k:3 * k] = 0.0
        cols["rot_1"][3 * k:3 * k + 5] = np.inf
        cols["rot_2"][3 * k + 5:3 * k + 10] = np.nan
        if rest:
            cols[rest[0]][:k] = rng.choice([1e5, -1e5, 1e-7, -3e-5, 65504.0, 65519.0, 65520.0], size=k)
    rows = [{nm: float(cols[nm][i]) if nm in cols else 0.0 for nm in names} for i in range(n)]
    for r in rows:
        for t, nm in props:
            if t not in ("float", "double", "float32", "float64"):
                lo, hi = {"b": (-128, 127), "B": (0, 255), "h": (-32768, 32767), "H": (0, 65535),
                          "i": (-2**31, 2**31 - 1), "I": (0, 2**32 - 1)}[FMT[t]]
                r[nm] = int(min(max(round(r[nm] * 8), lo), hi))
    return ply(props, rows)


def spz_bytes(n, version, file_degree, seed, fraction=12):
    """A .spz with random field bytes (every byte pattern is a valid splat)."""
    rng = np.random.default_rng(seed)
    head = struct.pack("<IIIBBBB", 0x5053474E, version, n, file_degree, fraction, 0, 0)
    pos = rng.integers(0, 256, size=n * (6 if version == 1 else 9), dtype=np.uint8)
    if version == 1:   # keep halves finite
        h = pos.view(np.uint16)
        h &= np.uint16(0xBBFF)
    coefs = [0, 3, 8, 15, 24][file_degree]
    parts = [pos, rng.integers(0, 256, n, dtype=np.uint8), rng.integers(0, 256, 3 * n, dtype=np.uint8),
             rng.integers(0, 256, 3 * n, dtype=np.uint8),
             rng.integers(0, 256, n * (4 if version >= 3 else 3), dtype=np.uint8),
             rng.integers(0, 256, n * coefs * 3, dtype=np.uint8)]
    return gzip.compress(head + b"".join(p.tobytes() for p in parts))


def colour_of(centers, i):
    w = int(centers[i:i + 1, 3].view(np.uint32)[0])
    return [w & 255, (w >> 8) & 255, (w >> 16) & 255, w >> 24]


def halves_of(sh, count):
    return sh.view(np.uint16)[:count].view(np.float16).astype(np.float64)


# ------------------------------------------------------------------ CPU

def test_reference_ply_case():
    props = float_props(["x", "y", "z", "nx", "ny", "nz", "f_dc_0", "f_dc_1", "f_dc_2", "opacity",
                         "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3"])
    c = O.parse_ply(ply(props, [
        {"x": -1, "y": 0, "z": 4, "f_dc_0": (1 - 0.5) / SH_C0, "f_dc_1": 0, "f_dc_2": (0 - 0.5) / SH_C0,
         "opacity": 0, "scale_0": math.log(2), "scale_1": math.log(3), "scale_2": 0, "rot_0": 2},
        {"x": 5, "y": -2, "z": 0, "rot_0": 1}]))
    assert c.count == 2 and c.degree == 0
    assert colour_of(c.centers, 0) == [255, 128, 0, 128]
    assert np.allclose(c.covariances[0][[0, 3, 5]], [4, 9, 1], rtol=1e-6)
    assert list(c.min) == [-1, -2, 0] and list(c.max) == [5, 0, 4]


def test_reference_ply_harmonics_case():
    rest = [f"f_rest_{k}" for k in range(9)]
    row = {"rot_0": 1}
    for k in range(3):
        row[f"f_rest_{k}"], row[f"f_rest_{k + 3}"], row[f"f_rest_{k + 6}"] = k, 10 + k, -(k + 1)
    c = O.parse_ply(ply(float_props(PLY_BASE + rest), [row, row]))
    assert c.degree == 1 and c.sh.size == 2 * 5 + 1
    h = halves_of(c.sh, 20)
    for i in (0, 1):
        for k in range(3):
            at = i * 10 + k * 3
            assert list(h[at:at + 3]) == [k, 10 + k, -(k + 1)]


@pytest.mark.parametrize("data,message", [
    (ply(float_props(PLY_BASE + ["f_rest_0", "f_rest_1"]), [{}]),
     "2 f_rest_ properties; harmonics of degree 1, 2 or 3 have 9, 24 or 45"),
    (ply(float_props(PLY_BASE), [{}], fmt="ascii"), "only binary_little_endian"),
    (ply(float_props(["x", "y", "z"]), [{}]), "not a splat capture: no f_dc_0"),
    (ply(float_props(PLY_BASE), [{}, {}])[:-4], "cut short"),
    (b"ply\nformat binary_little_endian 1.0\nelement chunk 4\nend_header\n", "a compressed .ply"),
    (b"ply\nformat binary_little_endian 1.0\nelement face 4\nend_header\n", "first element is 'face'"),
    (b"ply\nformat binary_little_endian 1.0\nelement vertex 1\n", "no end_header"),
    (b"ply\nformat binary_little_endian 1.0\nelement vertex 1\nproperty list uchar int v\nend_header\n",
     "list properties"),
    (b"ply\nformat binary_little_endian 1.0\nelement vertex 1\nproperty half x\nend_header\n",
     "unknown .ply property type 'half'"),
    (b"ply\nformat binary_little_endian 1.0\nelement vertex 1.5\nend_header\n", "a .ply with 1.5 vertices"),
    (ply(float_props(PLY_BASE), [{"x": float("nan")}, {}]), "splat 0 has a position that is not a number"),
])
def test_oracle_ply_refusals(data, message):
    with pytest.raises(O.OracleError, match=message.replace("(", r"\(").replace(")", r"\)").replace(".", r"\.")):
        O.parse_ply(data)


def test_pinned_exp_is_the_nearest_double():
    decimal.getcontext().prec = 60
    rng = np.random.default_rng(4)
    # normal results (x > ln 2^-1022); below that the pinned exp rounds twice
    xs = list(rng.uniform(-708.39, 709.7, 1500)) + list(rng.normal(0, 3, 1500)) + [0.0, 1.0, -1.0, math.log(2)]
    for x in xs:
        want = float(decimal.Decimal(float(x)).exp())
        assert O.lib().or_exp(float(x)) == want, x


def test_byte_and_half_rules():
    L = O.lib()
    assert L.or_byte(0.5 / 255) == 1 and L.or_byte(-0.001) == 0 and L.or_byte(2.0) == 255
    assert L.or_byte(float("nan")) == 0 and L.or_byte(1.5 / 255) == 2   # halves round up
    for v in (0.0, 1.0, -2.5, 65504.0, 65519.0, 1e9, 1e-8, 3e-6, -0.0):
        want = int(np.float16(np.clip(v, -65504, 65504)).view(np.uint16)) if abs(v) >= 2 ** -24 else 0
        if v < 0 and want == 0:
            want = 0x8000
        assert L.or_signed_half(v) == want, v


def test_hand_built_spz_splat():
    # one splat, version 2, fraction 12: position (1, 2, 3) in RUB -> (1, -2, -3);
    # rotation bytes (127.5 + 0 ...) -> identity-ish; scales 16 * (10 + ln 0.5) ...
    n = 1
    head = struct.pack("<IIIBBBB", 0x5053474E, 2, n, 0, 12, 0, 0)
    pos = b"".join(struct.pack("<i", v << 12)[:3] for v in (1, 2, 3))
    alpha = bytes([200])
    colour = bytes([round((0.5 * 0.15 + 0.5) * 255)] * 3)
    scales = bytes([160, 160, 160])            # exp(160 / 16 - 10) = 1
    rot = bytes([128, 128, 128])               # x = y = z = 1/255, w = sqrt(1 - 3/255^2)
    c = O.parse_spz(gzip.compress(head + pos + alpha + colour + scales + rot))
    assert list(c.centers[0, :3]) == [1, -2, -3]
    assert colour_of(c.centers, 0)[3] == 200
    assert np.allclose(c.covariances[0][[0, 3, 5]], [1, 1, 1], atol=1e-3)
    with pytest.raises(O.OracleError, match="gzipped, but not a .spz"):
        O.parse_spz(gzip.compress(b"\0" * 32))
    with pytest.raises(O.OracleError, match="cut short"):
        O.parse_spz(gzip.compress((head + pos)[:30]))
    with pytest.raises(O.OracleError, match="version 7"):
        O.parse_spz(gzip.compress(struct.pack("<IIIBBBB", 0x5053474E, 7, 1, 0, 12, 0, 0)))


# ------------------------------------------------------------------ GPU

def _check_same(sp, cap):
    centers, cov = sp.download()
    assert np.array_equal(centers.view(np.uint32), cap.centers.view(np.uint32))
    assert np.array_equal(cov.view(np.uint32), cap.covariances.view(np.uint32))
    assert list(sp.min) == list(cap.min) and list(sp.max) == list(cap.max)
    degree, words = sp.harmonics()
    assert degree == cap.degree
    if degree:
        assert np.array_equal(words, cap.sh[:words.size])


@pytest.mark.gpu
@pytest.mark.parametrize("degree", [0, 1, 2, 3])
def test_ply_matches_oracle(ctx, degree):
    from winding_b200 import load_splats
    data = random_ply(20_000, degree, seed=degree, extremes=True)
    sp = load_splats(data, ctx)
    try:
        _check_same(sp, O.parse_ply(data))
    finally:
        sp.destroy()


@pytest.mark.gpu
def test_ply_mixed_property_types(ctx):
    from winding_b200 import load_splats
    types = {"x": "double", "y": "double", "z": "float", "f_dc_0": "uchar", "f_dc_1": "short", "opacity": "char",
             "scale_0": "int", "rot_0": "ushort", "rot_1": "uint", "f_rest_4": "double"}
    data = random_ply(5000, 1, seed=9, types=types)
    sp = load_splats(data, ctx)
    try:
        _check_same(sp, O.parse_ply(data))
    finally:
        sp.destroy()


@pytest.mark.gpu
@pytest.mark.parametrize("version,file_degree", [(1, 0), (1, 1), (2, 2), (2, 4), (3, 3), (3, 0)])
def test_spz_matches_oracle(ctx, version, file_degree):
    from winding_b200 import load_splats
    data = spz_bytes(30_000, version, file_degree, seed=version * 10 + file_degree)
    sp = load_splats(data, ctx)
    try:
        _check_same(sp, O.parse_spz(data))
    finally:
        sp.destroy()


@pytest.mark.gpu
def test_loaded_ply_sorts_like_the_oracle(ctx):
    from winding_b200 import camera, load_splats, make_view
    data = random_ply(60_000, 0, seed=31)
    sp = load_splats(data, ctx)
    cap = O.parse_ply(data)
    try:
        mv = camera.look_at((0, 0, 60), (0, 0, 0))
        proj = camera.perspective(np.pi / 3, 1920 / 1080, 0.1)
        order, keys = ctx.sort(sp, make_view(mv, proj, (1920, 1080), 0.5))
        want_o, want_k = O.sort_view(cap, mv, proj, (1920.0, 1080.0), 0.5)
        assert np.array_equal(order, want_o) and np.array_equal(keys, want_k)
    finally:
        sp.destroy()


@pytest.mark.gpu
def test_load_refusals_and_splat_records(ctx):
    from winding_b200 import WsError, load_splats, parse_splats, workloads as W
    cases = [
        (ply(float_props(PLY_BASE + ["f_rest_0", "f_rest_1"]), [{}]), "2 f_rest_ properties"),
        (ply(float_props(PLY_BASE), [{}], fmt="ascii"), "only binary_little_endian"),
        (ply(float_props(["x", "y", "z"]), [{}]), "not a splat capture: no f_dc_0"),
        (ply(float_props(PLY_BASE), [{}, {}])[:-4], "cut short"),
        (b"ply\nformat binary_little_endian 1.0\nelement chunk 4\nend_header\n", "compressed .ply"),
        (ply(float_props(PLY_BASE), [{}, {}, {"y": float("inf")}, {"x": float("nan")}]),
         "splat 2 has a position that is not a number"),
        (b"PK\x03\x04" + b"\0" * 60, "a .sog needs decodeImage"),
        (b"NGSP" + struct.pack("<I", 4) + b"\0" * 24, "version 4, compressed with zstd"),
        (gzip.compress(b"\0" * 32), "gzipped, but not a .spz"),
        (gzip.compress(struct.pack("<IIIBBBB", 0x5053474E, 2, 5, 0, 12, 0, 0)), "the .spz is cut short"),
        (bytes(33), "not a whole number of 32-byte"),
    ]
    for data, message in cases:
        with pytest.raises(WsError, match=message.replace(".", r"\.").replace("(", r"\(")):
            load_splats(data, ctx)
    rec = W.uniform(3000, seed=5)
    a, b = load_splats(rec.tobytes(), ctx), parse_splats(rec, ctx)
    try:
        assert np.array_equal(a.download()[1], b.download()[1]) and a.degree == 0
    finally:
        a.destroy()
        b.destroy()
