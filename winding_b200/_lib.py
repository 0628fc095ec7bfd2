"""ctypes binding of libwsort.so (the C ABI in include/wsort.h).

There is no fallback: if the library is missing or does not load, importing
the functions that need it raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libwsort.so")

WS_OK = 0
WS_ERR_ARG = -1
WS_ERR_FORMAT = -2
WS_ERR_NAN = -3
WS_ERR_CAPACITY = -4
WS_ERR_CUDA = -5
WS_ERR_NOMEM = -6
WS_ERR_TIMEOUT = -7
WS_ERR_UNLOADED = -8
WS_ERR_BUSY = -9
WS_ERR_PENDING = -10

WS_HOST_OUTPUT = 0
WS_DEVICE_OUTPUT = 1
WS_MAX_SPLATS = 1 << 30
WS_NOALLOC_MAX_SPLATS = 1 << 20

ERROR_NAMES = {
    WS_ERR_ARG: "WS_ERR_ARG", WS_ERR_FORMAT: "WS_ERR_FORMAT", WS_ERR_NAN: "WS_ERR_NAN",
    WS_ERR_CAPACITY: "WS_ERR_CAPACITY", WS_ERR_CUDA: "WS_ERR_CUDA", WS_ERR_NOMEM: "WS_ERR_NOMEM",
    WS_ERR_TIMEOUT: "WS_ERR_TIMEOUT", WS_ERR_UNLOADED: "WS_ERR_UNLOADED", WS_ERR_BUSY: "WS_ERR_BUSY",
    WS_ERR_PENDING: "WS_ERR_PENDING",
}


class WsError(RuntimeError):
    """A failed call: `code` is the WS_ERR_* status, the message the library's text."""

    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code
        self.name = ERROR_NAMES.get(code, str(code))


class WsView(ctypes.Structure):
    _fields_ = [
        ("model_view", ctypes.c_float * 16),
        ("projection", ctypes.c_float * 16),
        ("viewport", ctypes.c_float * 2),
        ("cull", ctypes.c_float),
    ]


class WsJob(ctypes.Structure):
    _fields_ = [
        ("cloud", ctypes.c_void_p),
        ("view", WsView),
        ("order", ctypes.c_void_p),
        ("keys", ctypes.c_void_p),
        ("count", ctypes.c_void_p),
    ]


class WsEmitter(ctypes.Structure):
    _fields_ = [
        ("pool", ctypes.c_void_p),
        ("offset", ctypes.c_uint32),
        ("capacity", ctypes.c_uint32),
        ("eye", ctypes.c_float * 3),
        ("forward", ctypes.c_float * 3),
        ("order", ctypes.c_void_p),
        ("keys", ctypes.c_void_p),
        ("count", ctypes.c_void_p),
    ]


class WsShade(ctypes.Structure):
    _fields_ = [
        ("eye", ctypes.c_float * 3),
        ("reserved", ctypes.c_uint32),
        ("shaded", ctypes.c_void_p),
    ]


class WsParams(ctypes.Structure):
    _fields_ = [
        ("tile", ctypes.c_uint32),
        ("ctas_per_sm", ctypes.c_uint32),
        ("spin_limit", ctypes.c_uint32),
        ("segs_per_cta", ctypes.c_uint32),
        ("algorithm", ctypes.c_uint32),
    ]


ALGO_PHASES, ALGO_ONE_RADIX, ALGO_ONE_COUNT = 0, 1, 2
ONE_CTA_MAX = 16384   # largest job of splats the one-CTA sorts take


class WsServerOpts(ctypes.Structure):
    _fields_ = [
        ("memory_budget", ctypes.c_size_t),
        ("max_batch", ctypes.c_int),
        ("max_batch_splats", ctypes.c_uint64),
        ("streams", ctypes.c_int),
        ("queue_capacity", ctypes.c_int),
        ("collect_us", ctypes.c_int),
    ]


class WsImage(ctypes.Structure):
    _fields_ = [("width", ctypes.c_uint32), ("height", ctypes.c_uint32), ("rgba", ctypes.c_void_p)]


# int (*ws_decode_image)(void* user, const uint8_t* bytes, size_t nbytes, ws_image* out)
DECODE_IMAGE = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint8), ctypes.c_size_t,
                                ctypes.POINTER(WsImage))


class WsServerStats(ctypes.Structure):
    _fields_ = [
        ("submitted", ctypes.c_uint64),
        ("completed", ctypes.c_uint64),
        ("failed", ctypes.c_uint64),
        ("batches", ctypes.c_uint64),
        ("splats", ctypes.c_uint64),
        ("admission_waits", ctypes.c_uint64),
        ("in_flight", ctypes.c_uint64),
        ("peak_bytes", ctypes.c_uint64),
        ("p50_ms", ctypes.c_double),
        ("p99_ms", ctypes.c_double),
        ("mean_ms", ctypes.c_double),
        ("mean_batch", ctypes.c_double),
        ("max_batch_seen", ctypes.c_uint64),
        ("overlapped_batches", ctypes.c_uint64),
        ("cancelled", ctypes.c_uint64),
    ]


class WsTraceRec(ctypes.Structure):
    _fields_ = [
        ("claim_ns", ctypes.c_uint64),
        ("start_ns", ctypes.c_uint64),
        ("end_ns", ctypes.c_uint64),
        ("job", ctypes.c_uint32),
        ("phase", ctypes.c_uint32),
        ("segment", ctypes.c_uint32),
        ("sm", ctypes.c_uint32),
        ("mark_ns", ctypes.c_uint64 * 3),
    ]


vp = ctypes.c_void_p
u32p = ctypes.POINTER(ctypes.c_uint32)
f32p = ctypes.POINTER(ctypes.c_float)
f64p = ctypes.POINTER(ctypes.c_double)

# name -> (restype, argtypes); every symbol include/wsort.h declares.
SIGNATURES = {
    "ws_create": (ctypes.c_int, [ctypes.POINTER(vp), ctypes.c_int]),
    "ws_destroy": (ctypes.c_int, [vp]),
    "ws_last_error": (ctypes.c_char_p, [vp]),
    "ws_sync": (ctypes.c_int, [vp]),
    "ws_cloud_from_splat": (ctypes.c_int, [vp, ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(vp)]),
    "ws_cloud_from_device": (ctypes.c_int, [vp, vp, ctypes.c_size_t, ctypes.POINTER(vp)]),
    "ws_cloud_info": (ctypes.c_int, [vp, u32p, f64p, f64p]),
    "ws_cloud_download": (ctypes.c_int, [vp, vp, vp]),
    "ws_cloud_free": (ctypes.c_int, [vp]),
    "ws_depth_range": (ctypes.c_int, [vp, f32p, ctypes.POINTER(ctypes.c_int), f32p, f32p]),
    "ws_sort": (ctypes.c_int, [vp, vp, ctypes.POINTER(WsView), vp, vp, vp, ctypes.c_int, vp]),
    "ws_sort_batch": (ctypes.c_int, [vp, ctypes.c_int, ctypes.POINTER(WsJob), vp]),
    "ws_sort_batch_host": (ctypes.c_int, [vp, ctypes.c_int, ctypes.POINTER(WsJob), vp]),
    "ws_plan_create": (ctypes.c_int, [vp, ctypes.c_int, ctypes.POINTER(WsJob), ctypes.POINTER(vp)]),
    "ws_plan_set_views": (ctypes.c_int, [vp, ctypes.POINTER(WsView)]),
    "ws_plan_launch": (ctypes.c_int, [vp, vp]),
    "ws_plan_destroy": (ctypes.c_int, [vp]),
    "ws_device_alloc": (ctypes.c_int, [vp, ctypes.c_size_t, ctypes.POINTER(vp)]),
    "ws_device_free": (ctypes.c_int, [vp, vp]),
    "ws_device_download": (ctypes.c_int, [vp, vp, vp, ctypes.c_size_t, vp]),
    "ws_get_params": (ctypes.c_int, [vp, ctypes.POINTER(WsParams)]),
    "ws_set_params": (ctypes.c_int, [vp, ctypes.POINTER(WsParams)]),
    "ws_sort_noalloc": (ctypes.c_int, [vp, ctypes.POINTER(WsView), vp, vp, vp, vp]),
    "ws_sort_particles": (ctypes.c_int, [vp, ctypes.c_int, ctypes.POINTER(WsEmitter), vp]),
    "ws_cloud_set_harmonics": (ctypes.c_int, [vp, ctypes.c_int, vp, ctypes.c_size_t, ctypes.c_int]),
    "ws_cloud_load": (ctypes.c_int, [vp, vp, ctypes.c_size_t, ctypes.POINTER(ctypes.c_void_p)]),
    "ws_draw": (ctypes.c_int, [vp, vp, ctypes.POINTER(WsView), vp, vp, vp, vp, ctypes.c_uint32, ctypes.c_uint32, vp]),
    "ws_draw_tables": (ctypes.c_int, [ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]),
    "ws_set_draw_crowded": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32]),
    "ws_selftest_wait": (ctypes.c_int, [vp, ctypes.c_uint32]),
    "ws_selftest_noalloc_wait": (ctypes.c_int, [vp, ctypes.c_uint32, vp, vp]),
    "ws_inject_alloc_failures": (ctypes.c_int, [ctypes.c_int]),
    "ws_server_cancel": (ctypes.c_int, [vp, ctypes.c_uint64]),
    "ws_cloud_harmonics": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_int), vp]),
    "ws_cloud_read": (ctypes.c_int, [vp, vp, ctypes.c_size_t, vp, vp, ctypes.POINTER(ctypes.c_void_p)]),
    "ws_sort_batch_shaded": (ctypes.c_int, [vp, ctypes.c_int, ctypes.POINTER(WsJob), ctypes.POINTER(WsShade), vp]),
    "ws_particle_thresholds": (ctypes.c_int, [ctypes.POINTER(ctypes.c_float)]),
    "ws_server_create": (ctypes.c_int, [vp, ctypes.POINTER(WsServerOpts), ctypes.POINTER(vp)]),
    "ws_server_submit": (ctypes.c_int, [vp, vp, ctypes.POINTER(WsView), ctypes.POINTER(ctypes.c_uint64)]),
    "ws_server_poll": (ctypes.c_int, [vp, ctypes.c_uint64, ctypes.POINTER(ctypes.c_int)]),
    "ws_server_wait": (ctypes.c_int, [vp, ctypes.c_uint64, vp, vp, vp, ctypes.c_int]),
    "ws_server_result": (ctypes.c_int, [vp, ctypes.c_uint64, ctypes.POINTER(vp), ctypes.POINTER(vp),
                                        ctypes.POINTER(ctypes.c_uint32), ctypes.c_int]),
    "ws_server_release": (ctypes.c_int, [vp, ctypes.c_uint64]),
    "ws_server_get_stats": (ctypes.c_int, [vp, ctypes.POINTER(WsServerStats)]),
    "ws_server_destroy": (ctypes.c_int, [vp]),
    "ws_set_tuning": (ctypes.c_int, [vp, ctypes.POINTER(WsParams), ctypes.c_int]),
    "ws_copy_stats": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64),
                                     ctypes.c_int]),
    "ws_timing": (ctypes.c_int, [vp, ctypes.c_int]),
    "ws_timing_read": (ctypes.c_int, [vp, f64p, ctypes.POINTER(ctypes.c_uint64)]),
    "ws_trace": (ctypes.c_int, [vp, ctypes.c_int]),
    "ws_trace_read": (ctypes.c_int, [vp, ctypes.POINTER(WsTraceRec), ctypes.c_size_t,
                                     ctypes.POINTER(ctypes.c_size_t)]),
}

_lib = None


def load() -> ctypes.CDLL:
    """The loaded library. Raises OSError if libwsort.so is absent or broken:
    build it with `python -m winding_b200.build`."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"libwsort.so is not built ({LIB_PATH}); run python -m winding_b200.build")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int, ctx=None) -> None:
    if rc != WS_OK:
        msg = load().ws_last_error(ctx).decode() if ctx else ERROR_NAMES.get(rc, str(rc))
        raise WsError(rc, msg)
