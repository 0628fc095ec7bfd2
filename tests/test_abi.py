"""The C-ABI library loads and exports every function include/wsort.h
declares. No GPU needed: nothing here calls into CUDA."""
import ctypes
import os
import re

from winding_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"^\s*(?:const\s+)?\w+\*?\s+\*?(ws_\w+)\s*\(", text, flags=re.M))
    return names


def test_header_declares_the_sort_entry_points():
    names = declared_functions()
    for must in ("ws_create", "ws_cloud_from_splat", "ws_sort", "ws_sort_batch", "ws_plan_create"):
        assert must in names


def test_library_exports_every_declared_function():
    L = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in sorted(declared_functions()) if not hasattr(L, n)]
    assert not missing, missing


def test_binding_covers_every_declared_function():
    assert declared_functions() <= set(_lib.SIGNATURES), declared_functions() - set(_lib.SIGNATURES)


def test_view_struct_layout_matches_the_header():
    # float model_view[16], projection[16], viewport[2], cull
    assert ctypes.sizeof(_lib.WsView) == 35 * 4
    assert _lib.WsJob.view.offset == 8


def test_alloc_failure_hook_takes_counts_only():
    L = _lib.load()
    assert L.ws_inject_alloc_failures(-1) == _lib.WS_ERR_ARG
    assert L.ws_inject_alloc_failures(0) == _lib.WS_OK
