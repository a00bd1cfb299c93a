"""Degenerate and duplicated geometry through every variant: zero-area triangles and
segments, repeated primitives, collapsed edges, queries sitting on vertices and edge
midpoints.  The exact kernels must still match the oracle bit for bit; the fast forms
must agree with exact up to ties."""
import numpy as np
import pytest

import oracle
from gquery_b200 import _lib as L
from gquery_b200 import workloads as W
from gquery_b200.scene import Scene
from parity import REL_TOL, assert_bitwise, tie_report, to_np

pytestmark = pytest.mark.gpu


def _bad_mesh():
    v, f = W.icosphere(3, amplitude=0.2, seed=12)
    v = v.copy()
    f = f.copy()
    f[10] = [f[10][0], f[10][0], f[10][1]]        # repeated vertex: zero area
    v[f[20][2]] = v[f[20][1]]                       # collapsed edge in several faces
    dup = f[30:60].copy()                           # repeated faces
    col = np.array([[f[5][0], f[5][1], f[5][1]]])   # a segment-like triangle
    return v, np.concatenate([f, dup, col]).astype(np.int32)


def _queries(v, n, seed):
    rng = np.random.default_rng(seed)
    on_vertices = v[rng.integers(0, len(v), n // 4)]
    mids = 0.5 * (v[rng.integers(0, len(v), n // 4)] + v[rng.integers(0, len(v), n // 4)])
    near = v[rng.integers(0, len(v), n // 4)] * 1.01
    free = rng.uniform(-2, 2, size=(n - 3 * (n // 4), 3))
    return np.concatenate([on_vertices, mids, near, free]).astype(np.float32)


def test_degenerate_mesh_all_variants():
    v, f = _bad_mesh()
    s = Scene(v, f, 3, device=0, build_snch=True)
    q = _queries(v, 8000, 1)
    o, d = W.rays(8000, 3, seed=2)
    exact_cp = to_np(s.closest_point(q, variant="exact"))
    assert_bitwise(exact_cp, oracle.closest_point(3, s.ref_array(L.ARRAY_BVH_NODES), s.ref_array(L.ARRAY_PRIMITIVES), q),
                   ["valid", "p", "n", "uv", "d", "prim_id"], "cp ")
    exact_ray = to_np(s.intersect(o, d, variant="exact"))
    assert_bitwise(exact_ray, oracle.intersect(3, s.ref_array(L.ARRAY_BVH_NODES), s.ref_array(L.ARRAY_PRIMITIVES), o, d),
                   ["valid", "p", "d", "prim_id"], "ray ")
    exact_sil = to_np(s.closest_silhouette(q, variant="exact"))
    assert_bitwise(exact_sil,
                   oracle.closest_silhouette(3, s.ref_array(L.ARRAY_SNCH_NODES), s.ref_array(L.ARRAY_SILHOUETTES), q),
                   ["valid", "p", "d", "prim_id"], "sil ")
    for variant in ("coherent", "wide8"):
        rep = tie_report(exact_cp, to_np(s.closest_point(q, variant=variant)))
        assert rep["valid_mismatch"] == 0 and rep["prim_mismatch_not_tie"] == 0 and rep["max_rel_d"] <= REL_TOL, (
            variant, rep)
    rep = tie_report(exact_ray, to_np(s.intersect(o, d, variant="wide8")))
    assert rep["valid_mismatch"] == 0 and rep["prim_mismatch_not_tie"] == 0, rep
    for variant in ("coherent", "warp"):
        rep = tie_report(exact_sil, to_np(s.closest_silhouette(q, variant=variant)))
        assert rep["valid_mismatch"] == 0 and rep["prim_mismatch_not_tie"] == 0 and rep["max_rel_d"] <= REL_TOL, (
            variant, rep)
    assert s.device_error() == 0


def test_degenerate_polyline_all_variants():
    v, e = W.star_polyline(500, seed=3)
    v = v.copy()
    v[7] = v[6]                                     # zero-length segment
    e = np.concatenate([e, e[100:140], [[3, 3]]]).astype(np.int32)  # repeats and a point segment
    s = Scene(v, e, 2, device=0, build_snch=True)
    rng = np.random.default_rng(4)
    q = np.concatenate([v[rng.integers(0, len(v), 1000)], rng.uniform(-2, 2, (3000, 2))]).astype(np.float32)
    o, d = W.rays(4000, 2, seed=5)
    exact_cp = to_np(s.closest_point(q, variant="exact"))
    assert_bitwise(exact_cp, oracle.closest_point(2, s.ref_array(L.ARRAY_BVH_NODES), s.ref_array(L.ARRAY_PRIMITIVES), q),
                   ["valid", "p", "n", "t", "d", "prim_id"], "cp2 ")
    for variant in ("coherent", "wide8"):
        rep = tie_report(exact_cp, to_np(s.closest_point(q, variant=variant)))
        assert rep["valid_mismatch"] == 0 and rep["prim_mismatch_not_tie"] == 0 and rep["max_rel_d"] <= REL_TOL, (
            variant, rep)
    exact_ray = to_np(s.intersect(o, d, variant="exact"))
    rep = tie_report(exact_ray, to_np(s.intersect(o, d, variant="wide8")))
    assert rep["valid_mismatch"] == 0 and rep["prim_mismatch_not_tie"] == 0, rep
    exact_sil = to_np(s.closest_silhouette(q, variant="exact"))
    for variant in ("coherent", "warp"):
        rep = tie_report(exact_sil, to_np(s.closest_silhouette(q, variant=variant)))
        assert rep["valid_mismatch"] == 0 and rep["prim_mismatch_not_tie"] == 0, (variant, rep)
    assert s.device_error() == 0
