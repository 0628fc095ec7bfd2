"""Python front end of the request loop (ws_server_* in include/wsort.h).

    with Server(ctx, memory_budget=4 << 30) as srv:
        t = srv.submit(splats, view)          # from any thread
        order, keys = srv.wait(t)

Requests are batched continuously on the device: whatever has arrived when a
launch slot frees up goes into one persistent launch, in arrival order, as far
as the memory budget allows. Each result is identical to Context.sort's.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import WsError, WsServerOpts, WsServerStats
from .splats import Context, Splats


class Server:
    def __init__(self, ctx: Context, memory_budget: int = 0, max_batch: int = 0, max_batch_splats: int = 0,
                 streams: int = 0, queue_capacity: int = 0, collect_us: int = 0):
        self.ctx = ctx
        self.lib = ctx.lib
        opts = WsServerOpts(memory_budget, max_batch, max_batch_splats, streams, queue_capacity, collect_us)
        self.handle = ctypes.c_void_p()
        rc = self.lib.ws_server_create(ctx.handle, ctypes.byref(opts), ctypes.byref(self.handle))
        if rc != _lib.WS_OK:
            raise WsError(rc, f"ws_server_create failed ({_lib.ERROR_NAMES.get(rc, rc)})")
        self._counts: dict[int, int] = {}

    def submit(self, splats: Splats, view) -> int:
        t = ctypes.c_uint64()
        rc = self.lib.ws_server_submit(self.handle, splats.handle, ctypes.byref(view), ctypes.byref(t))
        if rc != _lib.WS_OK:
            raise WsError(rc, f"ws_server_submit: {_lib.ERROR_NAMES.get(rc, rc)}")
        self._counts[t.value] = splats.count
        return t.value

    def poll(self, ticket: int) -> bool:
        done = ctypes.c_int()
        rc = self.lib.ws_server_poll(self.handle, ticket, ctypes.byref(done))
        if rc != _lib.WS_OK:
            raise WsError(rc, f"ws_server_poll: {_lib.ERROR_NAMES.get(rc, rc)}")
        return bool(done.value)

    def wait(self, ticket: int, keys: bool = True, timeout_ms: int = -1):
        """(order, keys) host arrays of the request's survivors; releases it."""
        n = max(self._counts.get(ticket, 1), 1)
        order = np.empty(n, np.uint32)
        karr = np.empty(n, np.uint32) if keys else None
        count = ctypes.c_uint32()
        rc = self.lib.ws_server_wait(self.handle, ticket, order.ctypes.data, karr.ctypes.data if keys else None,
                                     ctypes.byref(count), timeout_ms)
        if rc != _lib.WS_OK:
            raise WsError(rc, f"ws_server_wait: {_lib.ERROR_NAMES.get(rc, rc)}")
        self._counts.pop(ticket, None)
        s = count.value
        return order[:s], (karr[:s] if keys else None)

    def result(self, ticket: int, timeout_ms: int = -1):
        """(order device pointer, keys device pointer, count): the result stays
        on the device until release(ticket)."""
        o = ctypes.c_void_p()
        k = ctypes.c_void_p()
        count = ctypes.c_uint32()
        rc = self.lib.ws_server_result(self.handle, ticket, ctypes.byref(o), ctypes.byref(k), ctypes.byref(count),
                                       timeout_ms)
        if rc != _lib.WS_OK:
            raise WsError(rc, f"ws_server_result: {_lib.ERROR_NAMES.get(rc, rc)}")
        return o.value, k.value, count.value

    def cancel(self, ticket: int) -> bool:
        """Withdraws a request still queued; False once it has been dispatched."""
        rc = self.lib.ws_server_cancel(self.handle, ticket)
        if rc == _lib.WS_ERR_BUSY:
            return False
        _lib.check(rc)
        return True

    def release(self, ticket: int) -> None:
        rc = self.lib.ws_server_release(self.handle, ticket)
        if rc != _lib.WS_OK:
            raise WsError(rc, f"ws_server_release: {_lib.ERROR_NAMES.get(rc, rc)}")
        self._counts.pop(ticket, None)

    def stats(self) -> dict:
        st = WsServerStats()
        rc = self.lib.ws_server_get_stats(self.handle, ctypes.byref(st))
        if rc != _lib.WS_OK:
            raise WsError(rc, "ws_server_get_stats")
        return {name: getattr(st, name) for name, _ in WsServerStats._fields_}

    def close(self) -> None:
        if self.handle:
            self.lib.ws_server_destroy(self.handle)
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
