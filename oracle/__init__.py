"""ORACLE — test infrastructure only (used by tests/, the smoke check and the
CPU-baseline leg of bench.py; never by the product).

ctypes wrapper of oracle/_build/liboracle.so, the scalar C++ restatement of the
reference traversals (see gq_oracle.cpp for the citations and the parity status).
Inputs are the reference float layouts (node / primitive / silhouette arrays),
queries are [n, D] float32.  Results come back as dicts of numpy arrays with the
record field names; misses are all-zero records like the reference's dr.zeros.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"
_lib = None


def build(force: bool = False) -> Path:
    srcs = [HERE / "gq_oracle.cpp", HERE.parent / "gquery_b200" / "csrc" / "gq_fmath.h"]
    if force or not LIB.exists() or any(s.stat().st_mtime > LIB.stat().st_mtime for s in srcs):
        subprocess.run(["make", "-C", str(HERE), "-B" if force else "all"], check=True, capture_output=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(str(LIB))
    return _lib


def n_threads() -> int:
    return int(os.environ.get("GQ_ORACLE_THREADS", "0")) or os.cpu_count() or 1


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _split(dim, kind, f, i):
    """Record fields from the oracle's row layout."""
    out = {"valid": i[:, 0] == 1, "prim_id": i[:, 1].copy(), "error": i[:, 0] < 0}
    if kind == "cp":
        out["p"] = f[:, 0:dim].T.copy()
        out["n"] = f[:, dim:2 * dim].T.copy()
        if dim == 2:
            out["t"] = f[:, 4].copy()
            out["d"] = f[:, 5].copy()
        else:
            out["uv"] = f[:, 6:8].T.copy()
            out["d"] = f[:, 8].copy()
    elif kind == "ray":
        out["p"] = f[:, 0:dim].T.copy()
        out["n"] = f[:, dim:2 * dim].T.copy()
        if dim == 2:
            out["t"] = f[:, 4].copy()
            out["d"] = f[:, 5].copy()
        else:
            out["uv"] = f[:, 6:8].T.copy()
            out["d"] = f[:, 8].copy()
        out["on_boundary"] = i[:, 2] == 1
    else:
        out["p"] = f[:, 0:dim].T.copy()
        out["d"] = f[:, dim].copy()
    return out


_KF = {("cp", 2): 6, ("cp", 3): 9, ("ray", 2): 6, ("ray", 3): 9, ("sil", 2): 3, ("sil", 3): 4}


def _run(name, kind, dim, args, nq, counts, threads, with_counts=True):
    f = np.zeros((nq, _KF[(kind, dim)]), np.float32)
    i = np.zeros((nq, 3), np.int32)
    cnt = np.zeros((nq, 2), np.int32) if counts else None
    fn = getattr(lib(), name)
    fn.restype = None
    cargs = []
    for a in args:
        if a is None:
            cargs.append(C.c_void_p(None))
        elif isinstance(a, np.ndarray):
            cargs.append(C.c_void_p(a.ctypes.data))
        else:
            cargs.append(C.c_int64(a))
    tail = [C.c_void_p(cnt.ctypes.data) if counts else C.c_void_p(None)] if with_counts else []
    fn(*cargs, C.c_void_p(f.ctypes.data), C.c_void_p(i.ctypes.data), *tail, C.c_int(threads or n_threads()))
    out = _split(dim, kind, f, i)
    if counts:
        out["interior"] = cnt[:, 0].copy()
        out["tested"] = cnt[:, 1].copy()
    return out


def closest_point(dim, nodes, prims, q, counts=False, threads=0):
    """BVH.closest_point / BVH3D.closest_point over reference arrays."""
    nodes, prims, q = _f(nodes), _f(prims), _f(q).reshape(-1, dim)
    return _run(f"orc_cp{dim}d", "cp", dim, [nodes, prims, q, q.shape[0]], q.shape[0], counts, threads)


def intersect(dim, nodes, prims, x, v, r_max=None, counts=False, threads=0):
    """BVH.intersect / BVH3D.intersect over reference arrays."""
    nodes, prims = _f(nodes), _f(prims)
    x, v = _f(x).reshape(-1, dim), _f(v).reshape(-1, dim)
    rm = None if r_max is None else _f(np.broadcast_to(np.asarray(r_max, np.float32), (x.shape[0],)))
    return _run(f"orc_ray{dim}d", "ray", dim, [nodes, prims, x, v, rm, x.shape[0]], x.shape[0], counts, threads)


def closest_silhouette(dim, snch_nodes, silhouettes, x, r_max=None, counts=False, threads=0):
    """SNCH.closest_silhouette / SNCH3D.closest_silhouette over reference arrays."""
    nodes, sils = _f(snch_nodes), _f(silhouettes)
    x = _f(x).reshape(-1, dim)
    rm = None if r_max is None else _f(np.broadcast_to(np.asarray(r_max, np.float32), (x.shape[0],)))
    return _run(f"orc_sil{dim}d", "sil", dim, [nodes, sils, x, rm, x.shape[0]], x.shape[0], counts, threads)


def _raw(dim, verts, index):
    return _f(verts).reshape(-1, dim), np.ascontiguousarray(index, np.int32).reshape(-1, dim)


def closest_point_baseline(dim, verts, index, q, threads=0):
    """closest_point_baseline (polyline.py:175-209, mesh.py:91-117) in FP32: the first
    strictly nearest primitive of the raw list, its record as the traversals'."""
    verts, index = _raw(dim, verts, index)
    q = _f(q).reshape(-1, dim)
    return _run(f"orc_cp_brute{dim}d", "cp", dim, [verts, index, index.shape[0], q, q.shape[0]], q.shape[0], False,
                threads, with_counts=False)


def intersect_baseline(dim, verts, index, x, v, r_max=None, threads=0):
    """intersect_baseline (polyline.py:137-169, mesh.py:60-84) in FP32: the first
    strictly nearest hit within r_max; on_boundary is set on every hit."""
    verts, index = _raw(dim, verts, index)
    x, v = _f(x).reshape(-1, dim), _f(v).reshape(-1, dim)
    rm = None if r_max is None else _f(np.broadcast_to(np.asarray(r_max, np.float32), (x.shape[0],)))
    return _run(f"orc_ray_brute{dim}d", "ray", dim, [verts, index, index.shape[0], x, v, rm, x.shape[0]], x.shape[0],
                False, threads, with_counts=False)


def brute_closest_point(dim, verts, index, q, threads=0):
    """FP64 nearest distance and primitive (original order)."""
    verts, q = _f(verts).reshape(-1, dim), _f(q).reshape(-1, dim)
    index = np.ascontiguousarray(index, np.int32).reshape(-1, dim)
    d = np.zeros(q.shape[0], np.float64)
    ids = np.zeros(q.shape[0], np.int32)
    fn = getattr(lib(), f"orc_brute_cp{dim}d")
    fn.restype = None
    fn(C.c_void_p(verts.ctypes.data), C.c_void_p(index.ctypes.data), C.c_int64(index.shape[0]),
       C.c_void_p(q.ctypes.data), C.c_int64(q.shape[0]), C.c_void_p(d.ctypes.data), C.c_void_p(ids.ctypes.data),
       C.c_int(threads or n_threads()))
    return d, ids


def brute_intersect3d(verts, index, x, v, threads=0):
    verts = _f(verts).reshape(-1, 3)
    x, v = _f(x).reshape(-1, 3), _f(v).reshape(-1, 3)
    index = np.ascontiguousarray(index, np.int32).reshape(-1, 3)
    t = np.zeros(x.shape[0], np.float64)
    ids = np.zeros(x.shape[0], np.int32)
    fn = lib().orc_brute_ray3d
    fn.restype = None
    fn(C.c_void_p(verts.ctypes.data), C.c_void_p(index.ctypes.data), C.c_int64(index.shape[0]),
       C.c_void_p(x.ctypes.data), C.c_void_p(v.ctypes.data), C.c_int64(x.shape[0]), C.c_void_p(t.ctypes.data),
       C.c_void_p(ids.ctypes.data), C.c_int(threads or n_threads()))
    return t, ids


def closest_silhouette_brute(dim, x, r_max=None, threads=0, *, vertices=None, indices=None, raw_silhouettes=None):
    """closest_silhouette_baseline: the first strictly nearest silhouette of the shape's
    list.  2D: the Polyline list built from vertices [nv, 2] / indices [ne, 2]
    (Polyline.configure_silhouette); 3D: the raw edges in the reference's flat layout
    (build_flat_silhouette_edges, 19 floats per edge)."""
    x = _f(x).reshape(-1, dim)
    rm = None if r_max is None else _f(np.broadcast_to(np.asarray(r_max, np.float32), (x.shape[0],)))
    nq = x.shape[0]
    f = np.zeros((nq, _KF[("sil", dim)]), np.float32)
    i = np.zeros((nq, 3), np.int32)
    if dim == 2:
        v = _f(vertices).reshape(-1, 2)
        e = np.ascontiguousarray(indices, dtype=np.int32).reshape(-1, 2)
        fn = lib().orc_sil_brute2d
        args = [v, v.shape[0], e, e.shape[0], x, rm, nq]
    else:
        s = _f(raw_silhouettes).reshape(-1)
        fn = lib().orc_sil_brute3d
        args = [s, s.size // 19, x, rm, nq]
    fn.restype = None
    cargs = [C.c_void_p(None) if a is None else C.c_void_p(a.ctypes.data) if isinstance(a, np.ndarray)
             else C.c_int64(a) for a in args]
    fn(*cargs, C.c_void_p(f.ctypes.data), C.c_void_p(i.ctypes.data), C.c_int(threads or n_threads()))
    return _split(dim, "sil", f, i)


# ---- the reference's own builder (oracle/_ref, built by `make -C oracle ref`) ----

REF_LIB = HERE / "_ref" / "libgqref.so"
_ref_lib = None
REF_ARRAYS = {"bvh_nodes": 0, "primitives": 1, "snch_nodes": 2, "silhouettes": 3, "raw_silhouettes": 4}


def build_ref(reference=None):
    """Compiles gQuery's own builder sources from a checkout (GQ_REFERENCE, or the
    default below) into oracle/_ref/libgqref.so.  Returns the library path, or None when
    neither a checkout nor a built library is at hand."""
    ref = Path(reference or os.environ.get("GQ_REFERENCE") or "/root/reference")
    deps = [HERE / "ref_builder.cpp", HERE / "eigen_subset" / "Eigen" / "Dense", HERE / "Makefile"]
    if not (ref / "src" / "shapes" / "bvh.cpp").exists():
        return REF_LIB if REF_LIB.exists() else None
    if not REF_LIB.exists() or any(d.stat().st_mtime > REF_LIB.stat().st_mtime for d in deps):
        subprocess.run(["make", "-C", str(HERE), "ref", f"REF={ref}"], check=True, capture_output=True)
    return REF_LIB


def ref_lib():
    global _ref_lib
    if _ref_lib is None:
        if build_ref() is None:
            raise FileNotFoundError("oracle/_ref/libgqref.so is not built and no gQuery checkout was found")
        _ref_lib = C.CDLL(str(REF_LIB))
        _ref_lib.gqref_build.restype = C.c_void_p
        _ref_lib.gqref_array.restype = C.c_int64
        _ref_lib.gqref_array.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int64]
        _ref_lib.gqref_free.argtypes = [C.c_void_p]
        _ref_lib.gqref_error.restype = C.c_char_p
        _ref_lib.gqref_flat_silhouette_edges.restype = C.c_int64
    return _ref_lib


def reference_build(dim, vertices, indices, snch=True, max_prims_in_node=10):
    """The reference's BVH / SNCH (src/shapes/bvh.cpp, snch.cpp) built from its own
    sources: a dict of its flat float arrays (node_data, primitive_data, silhouette_data,
    raw_silhouette_data) under the names of REF_ARRAYS."""
    lib = ref_lib()
    v = _f(vertices).reshape(-1, dim)
    ix = np.ascontiguousarray(indices, np.int32).reshape(-1, dim)
    h = lib.gqref_build(C.c_int(dim), C.c_void_p(v.ctypes.data), C.c_int64(v.shape[0]), C.c_void_p(ix.ctypes.data),
                        C.c_int64(ix.shape[0]), C.c_int(max_prims_in_node), C.c_int(1 if snch else 0))
    if not h:
        raise RuntimeError(lib.gqref_error().decode())
    try:
        out = {}
        for name, which in REF_ARRAYS.items():
            n = lib.gqref_array(h, which, None, 0)
            if n < 0:
                continue
            a = np.empty(n, np.float32)
            lib.gqref_array(h, which, C.c_void_p(a.ctypes.data), n)
            out[name] = a
        return out
    finally:
        lib.gqref_free(h)


def reference_flat_silhouette_edges(vertices, indices):
    """build_flat_silhouette_edges (src/shapes/silhouette_edge.cpp:62-71) from the
    reference's own source."""
    lib = ref_lib()
    v = _f(vertices).reshape(-1, 3)
    ix = np.ascontiguousarray(indices, np.int32).reshape(-1, 3)
    args = [C.c_void_p(v.ctypes.data), C.c_int64(v.shape[0]), C.c_void_p(ix.ctypes.data), C.c_int64(ix.shape[0])]
    n = lib.gqref_flat_silhouette_edges(*args, None, C.c_int64(0))
    a = np.empty(n, np.float32)
    lib.gqref_flat_silhouette_edges(*args, C.c_void_p(a.ctypes.data), C.c_int64(n))
    return a
