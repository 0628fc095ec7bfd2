"""Python host side of the splat sort, mirroring the reference's interface.

The reference (winding-engine, JavaScript) reads a capture with parseSplats
(src/scene/splats.js:60-76), uploads it as a Splats object
(src/render/splats.js:389-416) and sorts it per frame in SplatPass
(src/render/splats.js:418-728): prepare() decides which clouds need sorting,
_encodeSort() dispatches the three sort kernels. Here the same steps run
through libwsort.so:

    ctx = Context()                          # SplatPass.create
    splats = parse_splats(data, ctx)         # parseSplats + new Splats
    order, keys = ctx.sort(splats, view)     # one cloud, one view
    sp = SplatPass(ctx)                      # per-frame driver
    sp.prepare([(splats, world)], camera, 1920, 1080); sp.sort()

Errors are WsError with the reference's messages where it has one.
"""
from __future__ import annotations

import ctypes
from typing import Iterable

import numpy as np

from . import _lib
from ._lib import WsError, WsJob, WsView, check
from .camera import mat4_multiply

SPLAT_CULL = 0.5          # render/splats.js:78
CLOUD_FLOATS = 37         # render/splats.js:66: what a sort depends on
BUCKETS = 65536


def _f32(a, n: int) -> np.ndarray:
    out = np.ascontiguousarray(np.asarray(a, np.float32).reshape(-1))
    if out.size != n:
        raise ValueError(f"expected {n} floats, got {out.size}")
    return out


def make_view(model_view, projection, viewport=(1920.0, 1080.0), cull: float = SPLAT_CULL) -> WsView:
    v = WsView()
    ctypes.memmove(v.model_view, _f32(model_view, 16).ctypes.data, 64)
    ctypes.memmove(v.projection, _f32(projection, 16).ctypes.data, 64)
    v.viewport[0] = float(np.float32(viewport[0]))
    v.viewport[1] = float(np.float32(viewport[1]))
    v.cull = float(np.float32(cull)) if np.isfinite(cull) else float(cull)
    return v


class Context:
    """A sort context on one CUDA device (SplatPass.create's role)."""

    def __init__(self, device: int = 0):
        self.lib = _lib.load()
        self.handle = ctypes.c_void_p()
        rc = self.lib.ws_create(ctypes.byref(self.handle), int(device))
        if rc != 0:
            raise WsError(rc, f"ws_create failed on device {device}")
        self.device = device

    def close(self) -> None:
        if self.handle:
            self.lib.ws_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, rc: int) -> None:
        check(rc, self.handle)

    def sync(self) -> None:
        self.check(self.lib.ws_sync(self.handle))

    @property
    def params(self) -> _lib.WsParams:
        p = _lib.WsParams()
        self.check(self.lib.ws_get_params(self.handle, ctypes.byref(p)))
        return p

    def set_params(self, tile=None, ctas_per_sm=None, spin_limit=None, segs_per_cta=None, algorithm=None) -> None:
        """Kernel parameters (ws_params): tile = the least splats a segment
        covers, ctas_per_sm = 1 (1024-thread CTAs) or 2 (512-thread),
        segs_per_cta = segments per resident CTA, spin_limit = polls before a
        device-side wait gives up, algorithm = 0 (three phases), 1 (one-CTA
        radix) or 2 (one-CTA counting) for launches of small jobs of splats."""
        p = self.params
        if algorithm is not None:
            p.algorithm = algorithm
        if tile is not None:
            p.tile = tile
        if ctas_per_sm is not None:
            p.ctas_per_sm = ctas_per_sm
        if spin_limit is not None:
            p.spin_limit = spin_limit
        if segs_per_cta is not None:
            p.segs_per_cta = segs_per_cta
        self.check(self.lib.ws_set_params(self.handle, ctypes.byref(p)))

    def load(self, data) -> "Splats":
        return parse_splats(data, self)

    def sort(self, splats: "Splats", view: WsView, keys: bool = True):
        """(order, keys) as uint32 host arrays of the survivors, back to front."""
        splats._check_alive()
        n = max(splats.count, 1)
        order = np.empty(n, np.uint32)
        karr = np.empty(n, np.uint32) if keys else None
        count = ctypes.c_uint32(0)
        self.check(self.lib.ws_sort(self.handle, splats.handle, ctypes.byref(view), order.ctypes.data,
                                    karr.ctypes.data if keys else None, ctypes.byref(count),
                                    _lib.WS_HOST_OUTPUT, None))
        s = count.value
        return order[:s], (karr[:s] if keys else None)

    def sort_device(self, splats: "Splats", view: WsView, order_ptr: int, keys_ptr: int | None, count_ptr: int,
                    stream: int | None = None) -> None:
        """Queues a sort whose outputs are device pointers (e.g. torch tensors' data_ptr())."""
        self.check(self.lib.ws_sort(self.handle, splats.handle, ctypes.byref(view), order_ptr, keys_ptr, count_ptr,
                                    _lib.WS_DEVICE_OUTPUT, stream))

    def sort_batch(self, jobs: list[tuple], stream: int | None = None) -> None:
        """jobs: (splats, view, order_ptr, keys_ptr or None, count_ptr) with device pointers."""
        arr = (WsJob * len(jobs))()
        for j, (sp, view, o, k, c) in enumerate(jobs):
            sp._check_alive()
            arr[j].cloud = sp.handle
            arr[j].view = view
            arr[j].order = o
            arr[j].keys = k
            arr[j].count = c
        self.check(self.lib.ws_sort_batch(self.handle, len(jobs), arr, stream))

    def sort_batch_host(self, jobs: list[tuple], stream: int | None = None) -> None:
        """jobs as sort_batch, with host pointers (pinned for the one-copy
        path): every job's count, order and keys (or None) filled on return
        (ws_sort_batch_host)."""
        arr = (WsJob * len(jobs))()
        for j, (sp, view, o, k, c) in enumerate(jobs):
            sp._check_alive()
            arr[j].cloud = sp.handle
            arr[j].view = view
            arr[j].order = o
            arr[j].keys = k
            arr[j].count = c
        self.check(self.lib.ws_sort_batch_host(self.handle, len(jobs), arr, stream))

    def sort_batch_shaded(self, jobs: list[tuple], shades: list[tuple], stream: int | None = None) -> None:
        """jobs as sort_batch; shades: per job (eye, shaded_ptr), the eye in
        the cloud's space and a device array of its cloud's count words that
        receives the survivors' shaded colours (ws_sort_batch_shaded)."""
        arr = (WsJob * len(jobs))()
        sh = (_lib.WsShade * len(jobs))()
        for j, ((sp, view, o, k, c), (eye, shaded)) in enumerate(zip(jobs, shades)):
            sp._check_alive()
            arr[j].cloud = sp.handle
            arr[j].view = view
            arr[j].order = o
            arr[j].keys = k
            arr[j].count = c
            sh[j].eye[:] = [float(np.float32(x)) for x in eye]
            sh[j].shaded = shaded
        self.check(self.lib.ws_sort_batch_shaded(self.handle, len(jobs), arr, sh, stream))

    def draw(self, splats: "Splats", view: WsView, order_ptr: int, count_ptr: int, image_ptr: int, width: int,
             height: int, shaded_ptr: int | None = None, stream: int | None = None) -> None:
        """Blends the first *count splats of a sort's order (device pointers)
        over an RGBA f32 device image of width x height (ws_draw)."""
        splats._check_alive()
        self.check(self.lib.ws_draw(self.handle, splats.handle, ctypes.byref(view), order_ptr, count_ptr,
                                    shaded_ptr, image_ptr, int(width), int(height), stream))

    def set_draw_crowded(self, min_splats: int) -> None:
        """Tiles whose splat list holds min_splats or more (a power of two;
        0: none) are blended with four warps to a row pair
        (ws_set_draw_crowded); the image is the same either way."""
        self.check(self.lib.ws_set_draw_crowded(self.handle, int(min_splats)))

    def sort_particles(self, emitters: list[tuple], stream: int | None = None) -> None:
        """emitters: (pool_ptr, offset, capacity, eye, forward, order_ptr,
        keys_ptr or None, count_ptr), pointers into device memory; one launch
        for all (ws_sort_particles)."""
        arr = (_lib.WsEmitter * max(len(emitters), 1))()
        for j, (pool, offset, capacity, eye, forward, o, k, c) in enumerate(emitters):
            arr[j].pool = pool
            arr[j].offset = offset
            arr[j].capacity = capacity
            arr[j].eye[:] = [float(np.float32(x)) for x in eye]
            arr[j].forward[:] = [float(np.float32(x)) for x in forward]
            arr[j].order = o
            arr[j].keys = k
            arr[j].count = c
        self.check(self.lib.ws_sort_particles(self.handle, len(emitters), arr, stream))

    def plan(self, jobs: list[tuple]) -> "Plan":
        return Plan(self, jobs)

    def timing(self, enable: bool = True) -> None:
        self.check(self.lib.ws_timing(self.handle, int(enable)))

    def timing_read(self) -> tuple[float, int]:
        """(summed sort-kernel ms, sort kernels launched) since the last read."""
        ms = ctypes.c_double()
        n = ctypes.c_uint64()
        self.check(self.lib.ws_timing_read(self.handle, ctypes.byref(ms), ctypes.byref(n)))
        return ms.value, n.value

    def copy_stats(self, reset: bool = False) -> tuple[int, int]:
        """(host-to-device, device-to-host) bytes the sort calls moved (ws_copy_stats)."""
        h = ctypes.c_uint64()
        d = ctypes.c_uint64()
        self.check(self.lib.ws_copy_stats(self.handle, ctypes.byref(h), ctypes.byref(d), int(reset)))
        return h.value, d.value

    def trace(self, enable: bool = True) -> None:
        self.check(self.lib.ws_trace(self.handle, int(enable)))

    def trace_read(self) -> np.ndarray:
        """The last traced launch's work items as a structured array
        (claim_ns, start_ns, end_ns, job, phase, segment, sm, mark_ns)."""
        n = ctypes.c_size_t()
        self.check(self.lib.ws_trace_read(self.handle, None, 0, ctypes.byref(n)))
        recs = (_lib.WsTraceRec * max(n.value, 1))()
        self.check(self.lib.ws_trace_read(self.handle, recs, n.value, ctypes.byref(n)))
        dt = np.dtype([("claim_ns", "<u8"), ("start_ns", "<u8"), ("end_ns", "<u8"), ("job", "<u4"),
                       ("phase", "<u4"), ("segment", "<u4"), ("sm", "<u4"), ("mark_ns", "<u8", (3,))])
        return np.frombuffer(bytes(recs), dtype=dt, count=n.value).copy()

    # device buffers, for callers without torch
    def alloc(self, nbytes: int) -> int:
        p = ctypes.c_void_p()
        self.check(self.lib.ws_device_alloc(self.handle, nbytes, ctypes.byref(p)))
        return p.value

    def free(self, ptr: int) -> None:
        self.check(self.lib.ws_device_free(self.handle, ptr))

    def download(self, ptr: int, nbytes: int, dtype=np.uint32, stream: int | None = None) -> np.ndarray:
        out = np.empty(max(nbytes, 4) // np.dtype(dtype).itemsize, dtype)
        self.check(self.lib.ws_device_download(self.handle, ptr, out.ctypes.data, nbytes, stream))
        return out[: nbytes // np.dtype(dtype).itemsize]


class Plan:
    """A batch frozen into a CUDA graph; views can change between launches."""

    def __init__(self, ctx: Context, jobs: list[tuple]):
        self.ctx = ctx
        arr = (WsJob * len(jobs))()
        for j, (sp, view, o, k, c) in enumerate(jobs):
            arr[j].cloud = sp.handle
            arr[j].view = view
            arr[j].order = o
            arr[j].keys = k
            arr[j].count = c
        self.handle = ctypes.c_void_p()
        self.n = len(jobs)
        ctx.check(ctx.lib.ws_plan_create(ctx.handle, len(jobs), arr, ctypes.byref(self.handle)))

    def set_views(self, views: list[WsView]) -> None:
        arr = (WsView * self.n)(*views)
        self.ctx.check(self.ctx.lib.ws_plan_set_views(self.handle, arr))

    def launch(self, stream: int | None = None) -> None:
        self.ctx.check(self.ctx.lib.ws_plan_launch(self.handle, stream))

    def close(self) -> None:
        if self.handle:
            self.ctx.lib.ws_plan_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Splats:
    """A capture resident on the device: count, min, max (src/render/splats.js:389-416)."""

    def __init__(self, ctx: Context, handle: ctypes.c_void_p):
        self.ctx = ctx
        self.handle = handle
        cnt = ctypes.c_uint32()
        lo = (ctypes.c_double * 3)()
        hi = (ctypes.c_double * 3)()
        ctx.check(ctx.lib.ws_cloud_info(handle, ctypes.byref(cnt), lo, hi))
        self.count = cnt.value
        self.min = [lo[0], lo[1], lo[2]]
        self.max = [hi[0], hi[1], hi[2]]
        self.unloaded = False
        self.degree = 0

    def _check_alive(self):
        if self.unloaded:
            raise WsError(_lib.WS_ERR_UNLOADED, "addSplats: these splats were unloaded; remove the node first")

    def download(self):
        """(centers f32[n,4], covariances f32[n,6]) as parseSplats returns them."""
        self._check_alive()
        c = np.empty((self.count, 4), np.float32)
        v = np.empty((self.count, 6), np.float32)
        self.ctx.check(self.ctx.lib.ws_cloud_download(self.handle, c.ctypes.data, v.ctypes.data))
        return c, v

    def depth_range(self, model_view):
        vis = ctypes.c_int()
        dmin = ctypes.c_float()
        dscale = ctypes.c_float()
        mv = _f32(model_view, 16)
        self.ctx.check(self.ctx.lib.ws_depth_range(self.handle, mv.ctypes.data_as(_lib.f32p), ctypes.byref(vis),
                                                   ctypes.byref(dmin), ctypes.byref(dscale)))
        return bool(vis.value), dmin.value, dscale.value

    def harmonics(self):
        """(degree, words): the higher harmonics the cloud holds, words as
        uint32 (SH_WORDS[degree] a splat), or (0, None)."""
        self._check_alive()
        d = ctypes.c_int(0)
        self.ctx.check(self.ctx.lib.ws_cloud_harmonics(self.handle, ctypes.byref(d), None))
        if d.value == 0:
            return 0, None
        words = np.empty(self.count * SH_WORDS[d.value], np.uint32)
        self.ctx.check(self.ctx.lib.ws_cloud_harmonics(self.handle, ctypes.byref(d), words.ctypes.data))
        return d.value, words

    def set_harmonics(self, degree: int, words) -> None:
        """Attaches higher harmonics of `degree` (1-3): uint32 words packed as
        the reference packs them (sh_words(degree) a splat, see SH_WORDS), or
        degree 0 to drop them."""
        self._check_alive()
        if degree == 0:
            self.ctx.check(self.ctx.lib.ws_cloud_set_harmonics(self.handle, 0, None, 0, 0))
            self.degree = 0
            return
        w = np.ascontiguousarray(words, np.uint32).reshape(-1)
        self.ctx.check(self.ctx.lib.ws_cloud_set_harmonics(self.handle, int(degree), w.ctypes.data, w.size, 0))
        self.degree = int(degree)

    def destroy(self) -> None:
        """Frees the device arrays. The handle stays refusable: a later sort of
        it raises the reference's 'unloaded' error."""
        if not self.unloaded:
            self.ctx.check(self.ctx.lib.ws_cloud_free(self.handle))
            self.unloaded = True


def draw_tables():
    """(srgb, reach): the draw's decodeSRGB and log tables, 256 f32 each."""
    srgb = np.zeros(256, np.float32)
    reach = np.zeros(256, np.float32)
    check(_lib.load().ws_draw_tables(srgb.ctypes.data_as(_lib.f32p), reach.ctypes.data_as(_lib.f32p)))
    return srgb, reach


# 32-bit words a splat's harmonics take, by degree (scene/splats.js:43-47).
SH_WORDS = (0, 5, 12, 23)


def eye_in_cloud(model_view) -> np.ndarray:
    """The eye in a cloud's own space, as the reference fills Cloud.eye
    (render/splats.js:585-586): where the inverse of the f32 model-view
    takes the view's origin, in doubles, stored as f32."""
    m = np.asarray(model_view, np.float32).astype(np.float64).reshape(4, 4).T   # column-major
    inv = np.linalg.inv(m)
    return inv[:3, 3].astype(np.float32)


def load_splats(data, ctx: Context | None = None) -> Splats:
    """readSplats + upload (src/scene/splats.js:78-90): a binary .ply, a
    gzipped .spz (versions 1-3) or .splat records, decoded on the device with
    their harmonics. Raises WsError with the reference's messages."""
    ctx = ctx or Context(0)
    buf = np.frombuffer(bytes(data), np.uint8) if not isinstance(data, np.ndarray) else \
        np.ascontiguousarray(data).view(np.uint8).reshape(-1)
    h = ctypes.c_void_p()
    ctx.check(ctx.lib.ws_cloud_load(ctx.handle, buf.ctypes.data, buf.size, ctypes.byref(h)))
    sp = Splats(ctx, h)
    d = ctypes.c_int(0)
    ctx.check(ctx.lib.ws_cloud_harmonics(h, ctypes.byref(d), None))
    sp.degree = d.value
    return sp


def read_splats(data, decode_image=None, ctx: Context | None = None) -> Splats:
    """readSplats(bytes, {decodeImage}) (src/scene/splats.js:85-92): as
    load_splats, and a .sog bundle too, its images decoded by
    decode_image(bytes) -> (width, height, rgba), rgba width x height x 4
    bytes as stored (the reference's decodeImage). Raises WsError with the
    reference's messages; an exception of decode_image is raised as is."""
    ctx = ctx or Context(0)
    buf = np.frombuffer(bytes(data), np.uint8) if not isinstance(data, np.ndarray) else \
        np.ascontiguousarray(data).view(np.uint8).reshape(-1)
    keep = []        # decoded pixels, alive until the call returns
    raised = []

    def trampoline(user, ptr, n, out):
        try:
            width, height, rgba = decode_image(ctypes.string_at(ptr, n))
            pixels = np.ascontiguousarray(np.frombuffer(bytes(rgba), np.uint8) if not isinstance(rgba, np.ndarray)
                                          else rgba.view(np.uint8).reshape(-1))
            if pixels.size < int(width) * int(height) * 4:
                raise ValueError(f"decode_image gave {pixels.size} bytes for {width} x {height} pixels")
            keep.append(pixels)
            out[0].width, out[0].height = int(width), int(height)
            out[0].rgba = pixels.ctypes.data
            return 0
        except BaseException as e:   # noqa: BLE001 - handed back to the caller below
            raised.append(e)
            return 1

    callback = _lib.DECODE_IMAGE(trampoline) if decode_image is not None else None
    h = ctypes.c_void_p()
    rc = ctx.lib.ws_cloud_read(ctx.handle, buf.ctypes.data, buf.size,
                               ctypes.cast(callback, ctypes.c_void_p) if callback else None, None, ctypes.byref(h))
    if raised:
        raise raised[0]
    ctx.check(rc)
    sp = Splats(ctx, h)
    d = ctypes.c_int(0)
    ctx.check(ctx.lib.ws_cloud_harmonics(h, ctypes.byref(d), None))
    sp.degree = d.value
    return sp


def parse_splats(data, ctx: Context | None = None) -> Splats:
    """parseSplats + upload: .splat bytes (bytes, bytearray, numpy uint8 or
    structured records) to a resident cloud. Refuses what the reference refuses."""
    ctx = ctx or Context()
    if isinstance(data, np.ndarray):
        buf = np.ascontiguousarray(data).view(np.uint8).reshape(-1)
        raw = buf.ctypes.data_as(ctypes.c_char_p)
        nbytes = buf.size
    else:
        raw = bytes(data)
        nbytes = len(raw)
    h = ctypes.c_void_p()
    ctx.check(ctx.lib.ws_cloud_from_splat(ctx.handle, raw, nbytes, ctypes.byref(h)))
    return Splats(ctx, h)


class _State:
    """A placed cloud's sort buffers and what it was last sorted for (_stateFor, :629-674)."""

    def __init__(self, ctx: Context, splats: Splats):
        self.splats = splats
        n = max(1, splats.count)
        self.order = ctx.alloc(n * 4)
        self.keys = ctx.alloc(n * 4)
        self.count = ctx.alloc(4)
        self.last = np.full(CLOUD_FLOATS, np.nan, np.float32)   # NaN matches nothing: the first frame sorts
        self.next = np.zeros(CLOUD_FLOATS, np.float32)
        self.cull = None
        self.view = None

    def free(self, ctx: Context) -> None:
        for p in (self.order, self.keys, self.count):
            ctx.free(p)


class SplatPass:
    """The per-frame driver of the reference (SplatPass, src/render/splats.js:418-728)."""

    def __init__(self, ctx: Context):
        self.ctx = ctx
        self._states: dict[int, _State] = {}
        self._items: list[tuple] = []
        self.count = 0
        self.sorted = 0
        self.cull = SPLAT_CULL
        self.unjittered = None

    def prepare(self, clouds: Iterable[tuple], camera, width: float, height: float) -> int:
        """clouds: (splats, world f32[16]) pairs. Mirrors prepare (:546-618):
        modelView in FP64 stored f32, the cloud skipped when wholly behind the
        camera, sorted again only when its 37 floats or the cull changed,
        clouds far first. Returns how many clouds are drawn."""
        cull = self.cull
        if not (isinstance(cull, (int, float)) and np.isfinite(cull) and cull >= 0):
            raise WsError(_lib.WS_ERR_ARG, f"splatCull must be 0 or more, got {cull}")
        self._items = []
        self.count = 0
        self.sorted = 0
        for splats, world in clouds:
            if splats.unloaded:
                raise WsError(_lib.WS_ERR_UNLOADED, "addSplats: these splats were unloaded; remove the node first")
            state = self._states.get(id(splats))
            if state is None or state.splats is not splats:
                state = _State(self.ctx, splats)
                self._states[id(splats)] = state
            mv = mat4_multiply(camera.view, world)
            visible, _, _ = splats.depth_range(mv)
            if not visible:
                continue
            key = np.zeros(CLOUD_FLOATS, np.float32)
            key[0:16] = mv
            key[16:32] = camera.projection if self.unjittered is None else self.unjittered
            key[32] = width
            key[33] = height
            _, dmin, dscale = splats.depth_range(mv)
            key[34] = dmin
            key[35] = dscale
            key[36] = np.uint32(splats.count).view(np.float32)
            sort = not np.array_equal(state.last.view(np.uint32), key.view(np.uint32)) or state.cull != cull
            state.cull = cull
            if sort:
                state.next = key
                self.sorted += 1
            state.view = make_view(mv, camera.projection, (width, height), cull)
            lo, hi = splats.min, splats.max
            cx, cy, cz = ((lo[k] + hi[k]) / 2 for k in range(3))
            m = [float(v) for v in mv]
            depth = -(m[2] * cx + m[6] * cy + m[10] * cz + m[14])
            self._items.append((state, sort, depth))
            self.count += splats.count
        self._items.sort(key=lambda it: -it[2])
        return len(self._items)

    def sort(self) -> None:
        """_encodeSort (:676-697): every cloud that needs it, in one launch."""
        jobs = []
        for state, sort, _ in self._items:
            if not sort:
                continue
            state.last = state.next.copy()
            jobs.append((state.splats, state.view, state.order, state.keys, state.count))
        if jobs:
            self.ctx.sort_batch(jobs)

    def results(self):
        """(order, keys) host arrays per drawn cloud, in draw order (far first)."""
        out = []
        for state, _, _ in self._items:
            s = int(self.ctx.download(state.count, 4)[0])
            out.append((self.ctx.download(state.order, s * 4), self.ctx.download(state.keys, s * 4)))
        return out

    def destroy(self) -> None:
        for state in self._states.values():
            state.free(self.ctx)
        self._states.clear()
