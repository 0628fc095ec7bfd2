"""winding_b200: the Gaussian-splat depth-key + stable counting sort of the
Winding engine, as sm_100a CUDA behind a C ABI (libwsort.so).

The compute path is the CUDA library; this package is its Python host side
(ctypes), mirroring the reference's parseSplats / Splats / SplatPass.
"""
from ._lib import WsError
from .splats import Context, Plan, SplatPass, Splats, load_splats, make_view, parse_splats, read_splats, SPLAT_CULL

__all__ = ["WsError", "Context", "Plan", "SplatPass", "Splats", "load_splats", "make_view", "parse_splats", "read_splats",
           "SPLAT_CULL"]
