"""ctypes binding of libgq.so (the C ABI declared in include/gq.h).

The library is built in-tree by ``gquery_b200.build_lib`` (``__graft_entry__.build``).
There is no fallback: if the shared library is missing, loading raises.
"""
from __future__ import annotations

import ctypes as C
import threading
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libgq.so"

GQ_OK = 0
GQ_ERR_INVALID = 1
GQ_ERR_CUDA = 2
GQ_ERR_NOMEM = 3
GQ_ERR_DEPTH = 4
GQ_ERR_DEVICE = 5
GQ_ERR_UNSUPPORTED = 6

VARIANT_EXACT = 0
VARIANT_WIDE8 = 1
VARIANT_AUTO = 2
VARIANT_COHERENT = 3
VARIANT_WARP = 4
VARIANT_WIDE16 = 5

KIND_CLOSEST_POINT = 0
KIND_INTERSECT = 1
KIND_SILHOUETTE = 2

ARRAY_BVH_NODES = 0
ARRAY_PRIMITIVES = 1
ARRAY_SNCH_NODES = 2
ARRAY_SILHOUETTES = 3
ARRAY_RAW_SILHOUETTES = 4
ARRAY_WIDE_NODES = 5
ARRAY_SNCH_PAIRS = 6
ARRAY_SIL_RECORDS = 7
ARRAY_WIDE16_BOUNDS = 8

DEVERR_STACK = 1

BATCH_CP_EXACT = 1
BATCH_RAY_EXACT = 2
BATCH_SIL_EXACT = 8
BATCH_SIL_WARP = 16
BATCH_CP_SPLIT = 32
BATCH_SIL_SPLIT = 64
BATCH_ERR_SCENE = 1 << 8
BATCH_ERR_NO_SNCH = 1 << 9
SERVER_PER_REQUEST = 4


class BuildOpts(C.Structure):
    _fields_ = [("max_prims_in_node", C.c_int32), ("n_threads", C.c_int32), ("build_snch", C.c_int32),
                ("build_wide", C.c_int32), ("device", C.c_int32), ("gpu_build", C.c_int32)]


class SceneInfo(C.Structure):
    _fields_ = [("dim", C.c_int32), ("n_vertices", C.c_int64), ("n_prims", C.c_int64), ("n_nodes", C.c_int64),
                ("n_wide_nodes", C.c_int64), ("n_silhouettes", C.c_int64), ("max_depth", C.c_int32),
                ("exact_stack", C.c_int32), ("wide_stack", C.c_int32), ("device_bytes", C.c_int64),
                ("bbox_lo", C.c_float * 3), ("bbox_hi", C.c_float * 3)]


class Vecs(C.Structure):
    _fields_ = [("ptr", C.c_void_p), ("comp_stride", C.c_int64), ("elem_stride", C.c_int64)]


class CpOut(C.Structure):
    _fields_ = [("valid", C.c_void_p), ("p", C.c_void_p), ("n", C.c_void_p), ("t", C.c_void_p),
                ("d", C.c_void_p), ("prim_id", C.c_void_p)]


class RayOut(C.Structure):
    _fields_ = [("valid", C.c_void_p), ("p", C.c_void_p), ("n", C.c_void_p), ("t", C.c_void_p),
                ("d", C.c_void_p), ("prim_id", C.c_void_p), ("on_boundary", C.c_void_p)]


class SilOut(C.Structure):
    _fields_ = [("valid", C.c_void_p), ("p", C.c_void_p), ("d", C.c_void_p), ("prim_id", C.c_void_p)]


class Tuning(C.Structure):
    _fields_ = [("variant", C.c_int32), ("packet", C.c_int32), ("sorted", C.c_int32), ("persist", C.c_int32),
                ("budget", C.c_int32), ("block", C.c_int32), ("stack", C.c_int32)]


class QueryOpts(C.Structure):
    _fields_ = [("variant", C.c_int32), ("sort", C.c_int32), ("order", C.c_void_p), ("scratch", C.c_void_p),
                ("scratch_bytes", C.c_int64)]


class ServerOpts(C.Structure):
    _fields_ = [("budget_bytes", C.c_int64), ("ring_queries", C.c_int64 * 3), ("step_queries", C.c_int64),
                ("max_inflight", C.c_int32), ("flags", C.c_int32), ("sil_share", C.c_float),
                ("sil_slots", C.c_int32), ("sil_step_queries", C.c_int64), ("large_queries", C.c_int64),
                ("large_slots", C.c_int32), ("large_share", C.c_float), ("copy_threads", C.c_int32)]


class Request(C.Structure):
    _fields_ = [("scene", C.c_int32), ("kind", C.c_int32), ("n", C.c_int64), ("a", C.c_void_p), ("b", C.c_void_p),
                ("r_max", C.c_void_p), ("cp_out", CpOut), ("ray_out", RayOut), ("sil_out", SilOut),
                ("tag", C.c_uint64)]


class Completion(C.Structure):
    _fields_ = [("tag", C.c_uint64), ("t_submit", C.c_double), ("t_admit", C.c_double), ("t_launch", C.c_double),
                ("t_done", C.c_double), ("n", C.c_int64), ("kind", C.c_int32), ("step", C.c_int32),
                ("status", C.c_int32)]


class ServerStats(C.Structure):
    _fields_ = [("requests_done", C.c_int64), ("queries_done", C.c_int64), ("steps", C.c_int64),
                ("admitted_bytes_peak", C.c_int64), ("device_bytes", C.c_int64), ("device_error", C.c_int32),
                ("large_queries", C.c_int64)]


class BatchQueries(C.Structure):
    _fields_ = [("n", C.c_int64), ("scene", C.c_void_p), ("a", Vecs), ("b", Vecs), ("r_max", C.c_void_p)]


# name -> (restype, argtypes); every exported symbol of include/gq.h
SIGNATURES = {
    "gq_last_error": (None, [C.c_char_p, C.c_int64]),
    "gq_status_string": (C.c_char_p, [C.c_int32]),
    "gq_scene_build_2d": (C.c_int32, [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.POINTER(BuildOpts),
                                      C.POINTER(C.c_void_p)]),
    "gq_scene_build_3d": (C.c_int32, [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.POINTER(BuildOpts),
                                      C.POINTER(C.c_void_p)]),
    "gq_scene_free": (C.c_int32, [C.c_void_p]),
    "gq_scene_save": (C.c_int32, [C.c_void_p, C.c_char_p]),
    "gq_scene_load": (C.c_int32, [C.c_char_p, C.c_int32, C.POINTER(C.c_void_p)]),
    "gq_scene_get_info": (C.c_int32, [C.c_void_p, C.POINTER(SceneInfo)]),
    "gq_scene_set_tuning": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(Tuning)]),
    "gq_scene_get_tuning": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(Tuning)]),
    "gq_scene_ref_array": (C.c_int32, [C.c_void_p, C.c_int32, C.c_void_p, C.c_int64, C.POINTER(C.c_int64)]),
    "gq_flat_silhouette_edges": (C.c_int32, [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64,
                                             C.POINTER(C.c_int64)]),
    "gq_flat_silhouette_edges_device": (C.c_int32, [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p,
                                                    C.c_int64, C.POINTER(C.c_int64), C.c_int32, C.c_void_p]),
    "gq_query_scratch_bytes": (C.c_int64, [C.c_int64]),
    "gq_order_scratch_bytes": (C.c_int64, [C.c_int64]),
    "gq_query_order": (C.c_int32, [C.c_void_p, Vecs, C.c_int64, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]),
    "gq_closest_point": (C.c_int32, [C.c_void_p, Vecs, C.c_int64, C.POINTER(CpOut), C.POINTER(QueryOpts),
                                     C.c_void_p]),
    "gq_noalloc_max_queries": (C.c_int64, []),
    "gq_closest_point_noalloc": (C.c_int32, [C.c_void_p, Vecs, C.c_int64, C.POINTER(CpOut), C.c_int32, C.c_int32,
                                             C.c_void_p]),
    "gq_intersect": (C.c_int32, [C.c_void_p, Vecs, Vecs, C.c_void_p, C.c_int64, C.POINTER(RayOut),
                                 C.POINTER(QueryOpts), C.c_void_p]),
    "gq_closest_silhouette": (C.c_int32, [C.c_void_p, Vecs, C.c_void_p, C.c_int64, C.POINTER(SilOut),
                                          C.POINTER(QueryOpts), C.c_void_p]),
    "gq_closest_point_brute": (C.c_int32, [C.c_void_p, Vecs, C.c_int64, C.POINTER(CpOut), C.c_void_p]),
    "gq_intersect_brute": (C.c_int32, [C.c_void_p, Vecs, Vecs, C.c_void_p, C.c_int64, C.POINTER(RayOut),
                                       C.c_void_p]),
    "gq_closest_silhouette_brute": (C.c_int32, [C.c_void_p, Vecs, C.c_void_p, C.c_int64, C.POINTER(SilOut),
                                                C.c_void_p]),
    "gq_brute_f64": (C.c_int32, [C.c_void_p, C.c_int32, Vecs, Vecs, C.c_int64, C.c_void_p, C.c_void_p,
                                 C.c_void_p]),
    "gq_scene_device_error": (C.c_int32, [C.c_void_p, C.c_void_p, C.POINTER(C.c_int32)]),
    "gq_scene_set_stack_limit": (C.c_int32, [C.c_void_p, C.c_int32]),
    "gq_read_probe": (C.c_int32, [C.c_void_p, C.c_int64, C.c_int32, C.c_void_p, C.c_void_p]),
    "gq_ray_order": (C.c_int32, [C.c_void_p, Vecs, Vecs, C.c_int64, C.c_int32, C.c_void_p, C.c_void_p, C.c_int64,
                                 C.c_void_p]),
    "gq_batch_create": (C.c_int32, [C.c_void_p, C.c_int32, C.c_int64, C.c_int32, C.POINTER(C.c_void_p)]),
    "gq_batch_free": (C.c_int32, [C.c_void_p]),
    "gq_batch_device_bytes": (C.c_int64, [C.c_void_p]),
    "gq_batch_run": (C.c_int32, [C.c_void_p, C.POINTER(BatchQueries), C.POINTER(CpOut), C.POINTER(BatchQueries),
                                 C.POINTER(RayOut), C.POINTER(BatchQueries), C.POINTER(SilOut), C.c_void_p]),
    "gq_batch_device_error": (C.c_int32, [C.c_void_p, C.c_void_p, C.POINTER(C.c_int32)]),
    "gq_server_clock": (C.c_double, []),
    "gq_server_create": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(ServerOpts), C.POINTER(C.c_void_p)]),
    "gq_server_free": (C.c_int32, [C.c_void_p]),
    "gq_server_submit": (C.c_int32, [C.c_void_p, C.POINTER(Request)]),
    "gq_server_poll": (C.c_int32, [C.c_void_p, C.POINTER(Completion), C.c_int64, C.POINTER(C.c_int64)]),
    "gq_server_wait_idle": (C.c_int32, [C.c_void_p, C.c_double]),
    "gq_server_get_stats": (C.c_int32, [C.c_void_p, C.POINTER(ServerStats)]),
    "gq_server_run_trace": (C.c_int32, [C.c_void_p, C.POINTER(Request), C.c_void_p, C.c_int64,
                                        C.POINTER(Completion), C.c_double]),
}

_lock = threading.Lock()
_lib = None


class GQError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[gq status {status}] {message}")
        self.status = status


def lib() -> C.CDLL:
    """Loads libgq.so once (raises if it was never built)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not LIB_PATH.exists():
                raise ImportError(f"{LIB_PATH} is missing: run gquery_b200.build_lib.build() "
                                  "(the engine has no non-native fallback)")
            h = C.CDLL(str(LIB_PATH))
            for name, (res, args) in SIGNATURES.items():
                f = getattr(h, name)
                f.restype = res
                f.argtypes = args
            _lib = h
    return _lib


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    lib().gq_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status: int) -> None:
    if status != GQ_OK:
        raise GQError(status, last_error())
