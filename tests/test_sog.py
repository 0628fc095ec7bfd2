""".sog bundles (readSplats with decodeImage, src/scene/splats.js:85-200).

CPU: the oracle on the reference's own case (test/splats.test.js:258-321: a
one-splat .sog reads as the .ply it was made from -- log positions, the
smallest-three rotation, the codebooks and the harmonics palette) and its
refusals (:323-329), and the container and meta.json checks.
GPU: ws_cloud_read against the oracle, bit for bit, on that case and on
random bundles (degrees 0-3, stored and deflated entries, rotations with and
without a tag, labels past the palette, a short colour codebook), the
refusals with the same messages, and a decoder's own exception.
"""
import json
import math
import re
import struct
import zlib

import numpy as np
import pytest

from oracle import oracle as O
from tests.test_formats import PLY_BASE, colour_of, float_props, halves_of, ply

SQRT2 = math.sqrt(2.0)


def js_round(x):   # Math.round: halves up
    return math.floor(x + 0.5)


def zip_bytes(files, deflate=(), zip64=(), method=None):
    """A zip of the given files as a .sog bundles them: local headers, the
    entries (stored, or raw-deflated for names in `deflate`), the directory
    and its end record; checksums left zero, as the reference's own test
    writer leaves them."""
    parts, directory, offset = [], [], 0
    for name, data in files.items():
        nb = name.encode()
        m = 8 if name in deflate else 0
        if method and name in method:
            m = method[name]
        body = data
        if m == 8:
            z = zlib.compressobj(9, zlib.DEFLATED, -15)
            body = z.compress(data) + z.flush()
        size = 0xFFFFFFFF if name in zip64 else len(body)
        local = struct.pack("<IHHHHHIIIHH", 0x04034B50, 20, 0, m, 0, 0, 0, len(body), len(data), len(nb), 0) + nb
        central = struct.pack("<IHHHHHHIIIHHHHHII", 0x02014B50, 20, 20, 0, m, 0, 0, 0, size, len(data), len(nb),
                              0, 0, 0, 0, 0, offset) + nb
        parts += [local, body]
        directory.append(central)
        offset += len(local) + len(body)
    cd = b"".join(directory)
    end = struct.pack("<IHHHHIIH", 0x06054B50, 0, 0, len(directory), len(directory), len(cd), offset, 0)
    return b"".join(parts) + cd + end


def json_image(rgba, width):
    """An "image" whose file is its pixels as JSON (the reference test's)."""
    rgba = list(int(v) for v in rgba)
    return json.dumps({"width": width, "height": len(rgba) // 4 // width, "rgba": rgba}).encode()


def decode_json_image(data):
    d = json.loads(bytes(data).decode())
    return d["width"], d["height"], np.array(d["rgba"], np.uint8)


def raw_image(rgba, width, height):
    """A binary stand-in for a lossless WebP: width, height, then the pixels."""
    return struct.pack("<II", width, height) + np.asarray(rgba, np.uint8).tobytes()


def decode_raw_image(data):
    data = bytes(data)
    w, h = struct.unpack("<II", data[:8])
    return w, h, np.frombuffer(data[8:], np.uint8)


# --------------------------------------------------------- the reference case

SCALE_BOOK = [-6 + k * 0.05 for k in range(256)]
COLOUR_BOOK = [-2 + k / 64 for k in range(256)]
SH_BOOK = [-1 + k / 128 for k in range(256)]
MINS, MAXS = [-1, -2, -1], [1, 2, 1]
POSITION = [1.5, -2.25, 0.75]
_q = [0.9, 0.3, -0.2, 0.25]
ROTATION = [v / math.sqrt(sum(c * c for c in _q)) for v in _q]   # w x y z, w the largest
SCALE_INDEX = [100, 120, 130]
COLOUR_INDEX = [140, 100, 70]
REST_INDEX = [[160, 64, 128], [128, 176, 128], [96, 128, 192]]   # [channel][coefficient]


def reference_case():
    log = lambda x: math.copysign(math.log(abs(x) + 1), x)
    stored = [js_round((log(x) - MINS[a]) / (MAXS[a] - MINS[a]) * 65535) for a, x in enumerate(POSITION)]
    quat_bytes = [js_round((c * SQRT2 + 1) / 2 * 255) for c in ROTATION[1:]]
    images = {
        "means_l.webp": [stored[0] & 255, stored[1] & 255, stored[2] & 255, 255],
        "means_u.webp": [stored[0] >> 8, stored[1] >> 8, stored[2] >> 8, 255],
        "quats.webp": quat_bytes + [252],
        "scales.webp": SCALE_INDEX + [255],
        "sh0.webp": COLOUR_INDEX + [200],
        "shN_labels.webp": [1, 0, 0, 255],   # palette entry 1
    }
    centroids = np.zeros(192 * 4, np.uint8)   # entry 1 is columns 3..5 of the 192-wide row
    for k in range(3):
        centroids[(3 + k) * 4:(4 + k) * 4] = [REST_INDEX[0][k], REST_INDEX[1][k], REST_INDEX[2][k], 255]
    meta = {
        "version": 2, "count": 1,
        "means": {"mins": MINS, "maxs": MAXS, "files": ["means_l.webp", "means_u.webp"]},
        "scales": {"codebook": SCALE_BOOK, "files": ["scales.webp"]},
        "quats": {"files": ["quats.webp"]},
        "sh0": {"codebook": COLOUR_BOOK, "files": ["sh0.webp"]},
        "shN": {"count": 2, "bands": 1, "codebook": SH_BOOK, "files": ["shN_centroids.webp", "shN_labels.webp"]},
    }
    files = {"meta.json": json.dumps(meta).encode()}
    files.update({name: json_image(px, 1) for name, px in images.items()})
    files["shN_centroids.webp"] = json_image(centroids, 192)
    return meta, files


def reference_ply():
    row = {"x": POSITION[0], "y": POSITION[1], "z": POSITION[2],
           "scale_0": SCALE_BOOK[100], "scale_1": SCALE_BOOK[120], "scale_2": SCALE_BOOK[130],
           "rot_0": ROTATION[0], "rot_1": ROTATION[1], "rot_2": ROTATION[2], "rot_3": ROTATION[3],
           "opacity": math.log(200 / 55), "f_dc_0": COLOUR_BOOK[140], "f_dc_1": COLOUR_BOOK[100],
           "f_dc_2": COLOUR_BOOK[70]}
    for c in range(3):
        for k in range(3):
            row[f"f_rest_{c * 3 + k}"] = SH_BOOK[REST_INDEX[c][k]]
    names = PLY_BASE[:3] + ["f_dc_0", "f_dc_1", "f_dc_2", "opacity", "scale_0", "scale_1", "scale_2",
                            "rot_0", "rot_1", "rot_2", "rot_3"] + [f"f_rest_{k}" for k in range(9)]
    return ply(float_props(names), [row])


def test_oracle_reads_the_reference_case_as_its_ply():
    _, files = reference_case()
    got = O.parse_sog(zip_bytes(files), decode_json_image)
    want = O.parse_ply(reference_ply())
    assert got.count == 1 and got.degree == 1
    assert np.allclose(got.centers[0, :3], want.centers[0, :3], atol=1e-3)
    assert colour_of(got.centers, 0) == colour_of(want.centers, 0)
    assert np.allclose(got.covariances[0], want.covariances[0], atol=0.03)   # three bytes of rotation: near
    assert np.array_equal(halves_of(got.sh, 9), halves_of(want.sh, 9))


def _refusals():
    meta, files = reference_case()
    cases = []
    bare = lambda m: zip_bytes({"meta.json": json.dumps(m).encode()})
    with_meta = lambda m: zip_bytes({**files, "meta.json": json.dumps(m).encode()})
    cases.append((zip_bytes(files), None, "a .sog needs decodeImage, for its WebP images"))
    cases.append((bare({"means": {}}), decode_json_image, "a .sog of version 1; version 2 is read"))
    cases.append((bare({**meta, "version": 3}), decode_json_image, "a .sog of version 3; version 2 is read"))
    cases.append((bare({**meta, "version": "2"}), decode_json_image, "a .sog of version 2; version 2 is read"))
    cases.append((bare(meta), decode_json_image, "the .sog has no means_l.webp"))
    cases.append((with_meta({**meta, "count": 0}), decode_json_image, "a .sog of 0 splats"))
    cases.append((with_meta({**meta, "count": 1.5}), decode_json_image, "a .sog of 1.5 splats"))
    cases.append((with_meta({**meta, "count": 2}), decode_json_image, "means_l.webp has 1 pixels, for 2 splats"))
    cases.append((with_meta({k: v for k, v in meta.items() if k != "quats"}), decode_json_image,
                  "the .sog's meta.json has no quats"))
    cases.append((with_meta({**meta, "scales": {"files": ["scales.webp"]}}), decode_json_image,
                  "the .sog's meta.json has no scales.codebook"))
    cases.append((with_meta({**meta, "shN": {**meta["shN"], "bands": 2}}), decode_json_image,
                  "the .sog's harmonic palette is 192 wide; 512 for degree 2"))
    cases.append((with_meta({**meta, "sh0": {**meta["sh0"], "codebook": None}}), decode_json_image,
                  "the .sog's meta.json has no sh0.codebook"))
    cases.append((with_meta({**meta, "means": {**meta["means"], "mins": []}}), decode_json_image,
                  "splat 0 has a position that is not a number"))
    cases.append((zip_bytes({**files, "meta.json": b"{version: 2}"}), decode_json_image,
                  "the .sog's meta.json is not JSON"))
    cases.append((zip_bytes(files, zip64={"quats.webp"}), decode_json_image, "a zip64 .sog is not read"))
    cases.append((zip_bytes(files, method={"sh0.webp": 12}), decode_json_image,
                  "sh0.webp is compressed with method 12; stored and deflate are read"))
    whole = zip_bytes(files)
    cases.append((whole[:-30], decode_json_image, "a zip with no end record: cut short?"))
    # The directory's offset moved one byte on: its first entry is damaged.
    end = whole.rindex(b"PK\x05\x06")
    at = struct.unpack("<I", whole[end + 16:end + 20])[0]
    cases.append((whole[:end + 16] + struct.pack("<I", at + 1) + whole[end + 20:], decode_json_image,
                  "a zip whose directory is damaged"))
    # An entry that claims more bytes than the file has.
    cut = bytearray(whole)
    first = whole.index(b"PK\x01\x02")
    cut[first + 20:first + 24] = struct.pack("<I", len(whole))
    cases.append((bytes(cut), decode_json_image, "the zip is cut short in meta.json"))
    return cases


@pytest.mark.parametrize("k", range(19))
def test_oracle_refusals(k):
    data, decoder, message = _refusals()[k]
    with pytest.raises(O.OracleError, match=re.escape(message)):
        O.parse_sog(data, decoder)


def test_oracle_reads_deflated_entries_alike():
    _, files = reference_case()
    a = O.parse_sog(zip_bytes(files), decode_json_image)
    b = O.parse_sog(zip_bytes(files, deflate=set(files)), decode_json_image)
    assert np.array_equal(a.centers.view(np.uint32), b.centers.view(np.uint32))
    assert np.array_equal(a.sh, b.sh)


def random_sog(n, degree, seed, deflate=False, short_colour_book=False):
    """A random bundle: every pixel byte uniform, rotation tags 248-255 (some
    without a rotation), labels up to past the palette's end."""
    rng = np.random.default_rng(seed)
    px = lambda: rng.integers(0, 256, size=n * 4, dtype=np.uint8)
    quats = px()
    quats[3::4] = rng.integers(248, 256, size=n)
    width = max(1, int(math.ceil(math.sqrt(n))))
    height = (n + width - 1) // width

    def image(p):   # pad to the image's pixels
        full = np.zeros(width * height * 4, np.uint8)
        full[:p.size] = p
        return raw_image(full, width, height)

    colour_book = rng.normal(0, 1.5, 200 if short_colour_book else 256).tolist()
    meta = {
        "version": 2, "count": n,
        "means": {"mins": rng.uniform(-4, -1, 3).tolist(), "maxs": rng.uniform(1, 4, 3).tolist(),
                  "files": ["means_l.webp", "means_u.webp"]},
        "scales": {"codebook": rng.normal(-4, 1, 256).tolist(), "files": ["scales.webp"]},
        "quats": {"files": ["quats.webp"]},
        "sh0": {"codebook": colour_book, "files": ["sh0.webp"]},
    }
    files = {"means_l.webp": image(px()), "means_u.webp": image(px()), "quats.webp": image(quats),
             "scales.webp": image(px()), "sh0.webp": image(px())}
    if degree:
        per = O.SH_COEFFICIENTS[degree]
        entries = 700
        labels = np.zeros(n * 4, np.uint8)
        lab = rng.integers(0, entries + 100, size=n)   # some past shN.count
        labels[0::4], labels[1::4] = lab & 255, lab >> 8
        rows = (entries + 63) // 64 - 1                # the last row left out: labels there read off the end
        palette = rng.integers(0, 256, size=64 * per * rows * 4, dtype=np.uint8)
        meta["shN"] = {"count": entries, "bands": degree, "codebook": rng.normal(0, 0.4, 256).tolist(),
                       "files": ["shN_centroids.webp", "shN_labels.webp"]}
        files["shN_centroids.webp"] = raw_image(palette, 64 * per, rows)
        files["shN_labels.webp"] = image(labels)
    files["meta.json"] = json.dumps(meta).encode()
    return zip_bytes(files, deflate=set(files) if deflate else ())


def test_oracle_random_bundle_is_finite_and_boxed():
    cap = O.parse_sog(random_sog(2000, 2, seed=3), decode_raw_image)
    assert cap.count == 2000 and cap.degree == 2
    assert np.isfinite(cap.centers[:, :3]).all()
    # the box is kept in doubles, the centres in f32
    assert np.allclose(cap.min, cap.centers[:, :3].min(axis=0), rtol=1e-6)
    assert np.allclose(cap.max, cap.centers[:, :3].max(axis=0), rtol=1e-6)


# ------------------------------------------------------------------ GPU

def _same(sp, cap):
    """Bit for bit, NaN against NaN (a NaN's payload is the machine's)."""
    centers, cov = sp.download()

    def same(a, b):
        a, b = np.asarray(a, np.float32), np.asarray(b, np.float32)
        return bool(((a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))).all())

    assert same(centers, cap.centers)
    assert same(cov, cap.covariances)
    assert list(sp.min) == list(cap.min) and list(sp.max) == list(cap.max)
    degree, words = sp.harmonics()
    assert degree == cap.degree
    if degree:
        assert np.array_equal(words, cap.sh[:words.size])


@pytest.mark.gpu
def test_reference_case_matches_oracle(ctx):
    from winding_b200 import read_splats
    _, files = reference_case()
    data = zip_bytes(files)
    sp = read_splats(data, decode_json_image, ctx)
    try:
        _same(sp, O.parse_sog(data, decode_json_image))
    finally:
        sp.destroy()


@pytest.mark.gpu
@pytest.mark.parametrize("degree,deflate,short", [(0, False, False), (1, True, False), (2, False, True),
                                                  (3, True, True)])
def test_random_bundles_match_oracle(ctx, degree, deflate, short):
    from winding_b200 import read_splats
    data = random_sog(30_000, degree, seed=40 + degree, deflate=deflate, short_colour_book=short)
    sp = read_splats(data, decode_raw_image, ctx)
    try:
        _same(sp, O.parse_sog(data, decode_raw_image))
    finally:
        sp.destroy()


@pytest.mark.gpu
def test_refusals_match_oracle(ctx):
    from winding_b200 import WsError, read_splats
    for data, decoder, message in _refusals():
        with pytest.raises(O.OracleError) as want:
            O.parse_sog(data, decoder)
        with pytest.raises(WsError) as got:
            read_splats(data, decoder, ctx)
        assert str(got.value) == str(want.value) and message in str(got.value)


@pytest.mark.gpu
def test_other_formats_and_a_failing_decoder(ctx):
    from winding_b200 import read_splats
    from winding_b200 import workloads as W
    rec = W.uniform(1000, 5)
    sp = read_splats(rec.tobytes(), decode_json_image, ctx)   # not a zip: read as the records they are
    try:
        assert sp.count == 1000
    finally:
        sp.destroy()
    _, files = reference_case()

    def broken(data):
        raise RuntimeError("not a WebP")

    with pytest.raises(RuntimeError, match="not a WebP"):
        read_splats(zip_bytes(files), broken, ctx)
