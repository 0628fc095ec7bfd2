"""The particle sort of alpha emitters, host side (render/particles.js).

Every emitter's particles live in one pool, 32 bytes a particle (position
xyz, age, velocity xyz, lifetime as f32, render/particles.js:51-56), each
emitter a ring of it (offset, capacity). An alpha emitter is drawn far to
near: its live slots, keyed by 12 bits of log2 depth, in order
(makeKeys / scanCounts / place, :197-243). Here each frame's alpha emitters
go to the library in one launch (Context.sort_particles ->
ws_sort_particles), and the result of each is its live slots in
(key, slot) order, the reference's order with ties broken by slot.

    eye, forward = view_of(camera_position, view_matrix)
    sort_emitters(ctx, pool_ptr, [(offset, capacity), ...], eye, forward, outs)
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

PARTICLE_BYTES = 32     # render/particles.js:41
BUCKETS = 4096          # :45
LOG_NEAR = -10          # :47
LOG_FAR = 20            # :48


def view_of(camera_position, view_matrix):
    """(eye, forward) as the reference writes its View uniform
    (render/particles.js:688-693): the camera position, and minus the third
    row of the column-major view matrix, both as f32."""
    v = np.asarray(view_matrix, np.float64).reshape(16)
    eye = np.asarray(camera_position, np.float32).reshape(3)
    forward = np.array([-v[2], -v[6], -v[10]], np.float32)
    return eye, forward


def thresholds() -> np.ndarray:
    """The 4096 depth thresholds the kernel compares with: t[b] is the least
    f32 depth whose bucket is b or more (t[0] = 0)."""
    out = np.zeros(BUCKETS, np.float32)
    rc = _lib.load().ws_particle_thresholds(out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
    if rc:
        raise _lib.WsError(rc, "ws_particle_thresholds failed")
    return out


def sort_emitters(ctx, pool_ptr: int, rings, eye, forward, outs, stream: int | None = None) -> None:
    """Queues the sort of every ring (offset, capacity) of the pool at
    `pool_ptr` (device, 16-byte aligned) for one view. outs: per ring,
    (order_ptr, keys_ptr or None, count_ptr) in device memory."""
    if len(rings) != len(outs):
        raise ValueError("one output triple per ring")
    ctx.sort_particles([(pool_ptr, int(off), int(cap), eye, forward, o, k, c)
                        for (off, cap), (o, k, c) in zip(rings, outs)], stream)
