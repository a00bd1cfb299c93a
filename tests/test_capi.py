"""C ABI checks that need no GPU: the library loads, exports every function that
include/gq.h declares, and reports errors as status codes with messages."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from gquery_b200 import _lib as L
from gquery_b200.scene import Scene

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"\b(gq_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_header_declares_the_abi():
    names = declared_functions()
    assert "gq_closest_point" in names and "gq_scene_build_3d" in names
    assert len(names) >= 15


def test_library_exports_every_declared_symbol():
    h = L.lib()
    missing = [n for n in declared_functions() if not hasattr(h, n)]
    assert not missing, missing


def test_python_binding_covers_every_symbol():
    assert set(declared_functions()) <= set(L.SIGNATURES)


def test_status_strings_and_last_error():
    assert L.lib().gq_status_string(L.GQ_OK) == b"ok"
    assert b"invalid" in L.lib().gq_status_string(L.GQ_ERR_INVALID)
    out = C.c_void_p()
    st = L.lib().gq_scene_build_3d(None, 0, None, 0, None, C.byref(out))
    assert st == L.GQ_ERR_INVALID
    assert "null" in L.last_error()


def test_queries_on_host_only_scene_are_unsupported():
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    f = np.array([[0, 1, 2]], np.int32)
    s = Scene(v, f, 3, device=None)
    vecs = L.Vecs(1, 1, 3)  # never dereferenced: the call is refused first
    out = L.CpOut()
    st = L.lib().gq_closest_point(s.handle, vecs, 4, C.byref(out), None, None)
    assert st == L.GQ_ERR_UNSUPPORTED
    assert "device copy" in L.last_error()


def test_zero_queries_is_a_noop():
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    s = Scene(v, np.array([[0, 1, 2]], np.int32), 3, device=None)
    out = L.CpOut()
    assert L.lib().gq_closest_point(s.handle, L.Vecs(None, 0, 0), 0, C.byref(out), None, None) == L.GQ_OK


def test_scratch_sizes_grow_with_n():
    a, b = L.lib().gq_query_scratch_bytes(1000), L.lib().gq_query_scratch_bytes(100000)
    assert 0 < a < b
    assert L.lib().gq_query_scratch_bytes(0) == 0


def test_scene_info():
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], np.float32)
    f = np.array([[0, 1, 2], [0, 1, 3], [1, 2, 3], [0, 2, 3]], np.int32)
    s = Scene(v, f, 3, device=None)
    assert s.info["n_prims"] == 4 and s.info["dim"] == 3
    assert s.info["n_nodes"] % 2 == 1 and s.info["n_nodes"] <= 7
    assert s.info["device_bytes"] == 0
