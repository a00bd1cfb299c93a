"""Oracle pins (CPU): the README examples of the reference (examples/example_2d.py,
examples/example_3d.py) with answers derived in FP64 from the reference formulas,
FP64 brute force on random scenes, and the reference's quirks."""
import math

import numpy as np
import pytest

import oracle
from gquery_b200 import gquery_ext as gx
from gquery_b200 import workloads as W

PENTAGON_V = np.array([[0.0, 0.0], [1.0, 0.0], [1.5, 1.0], [0.5, 1.5], [-0.5, 1.0]], np.float32)
PENTAGON_E = np.array([[0, 1], [1, 2], [2, 3], [3, 4], [4, 0]], np.int32)
ABS_TOL = 5e-7  # 2 ulp at |x| = 2, the scale of every test scene
TETRA_V = np.array([[0, 0, 0], [1, 0, 0], [0.5, 1, 0], [0.5, 0.5, 1]], np.float32)
TETRA_F = np.array([[0, 1, 2], [0, 1, 3], [1, 2, 3], [0, 2, 3]], np.int32)


def arrays2():
    b = gx.BVH(PENTAGON_V, PENTAGON_E)
    s = gx.SNCH(PENTAGON_V, PENTAGON_E)
    return b.node_data(), b.primitive_data(), s.node_data(), s.silhouette_data()


def arrays3():
    b = gx.BVH3D(TETRA_V, TETRA_F)
    s = gx.SNCH3D(TETRA_V, TETRA_F)
    return b.node_data(), b.primitive_data(), s.node_data(), s.silhouette_data()


def test_kat_2d_closest_point():
    N, P, _, _ = arrays2()
    r = oracle.closest_point(2, N, P, np.array([[0.8, 0.8]]))
    assert r["valid"][0] and r["prim_id"][0] == 2
    assert np.allclose(r["p"][:, 0], [1.02, 1.24], rtol=2e-6)
    assert math.isclose(r["t"][0], 0.48, rel_tol=2e-6)
    assert math.isclose(r["d"][0], 0.4919350, rel_tol=2e-6)


def test_kat_2d_ray():
    N, P, _, _ = arrays2()
    r = oracle.intersect(2, N, P, np.array([[0.8, 0.8]]), np.array([[1.0, 1.0]]))
    assert r["valid"][0] and r["prim_id"][0] == 2 and r["on_boundary"][0]
    assert math.isclose(r["d"][0], 0.3666667, rel_tol=2e-6)
    assert np.allclose(r["p"][:, 0], [1.1666667, 1.1666667], rtol=2e-6)
    assert r["t"][0] == -1.0


def test_kat_2d_silhouette():
    _, _, SN, SS = arrays2()
    r = oracle.closest_silhouette(2, SN, SS, np.array([[2.0, 0.5]]))
    assert r["valid"][0] and r["prim_id"][0] == 2
    assert np.allclose(r["p"][:, 0], [1.5, 1.0])
    assert math.isclose(r["d"][0], 0.7071068, rel_tol=2e-6)


def test_kat_3d_closest_point():
    N, P, _, _ = arrays3()
    r = oracle.closest_point(3, N, P, np.array([[0.6, 0.6, 0.6]]))
    assert r["valid"][0] and r["prim_id"][0] == 2
    assert np.allclose(r["p"][:, 0], [0.5619048, 0.5809524, 0.5904762], rtol=2e-6)
    assert math.isclose(r["d"][0], 0.0436436, rel_tol=1e-5)


def test_kat_3d_ray_miss_is_zero_record():
    N, P, _, _ = arrays3()
    r = oracle.intersect(3, N, P, np.array([[0.6, 0.6, 0.6]]), np.array([[1.0, 1.0, 1.0]]))
    assert not r["valid"][0]
    assert r["prim_id"][0] == 0 and r["d"][0] == 0 and not r["p"].any() and not r["on_boundary"][0]


def test_kat_3d_silhouette_and_zero_fourth_vertex():
    _, _, SN, SS = arrays3()
    r = oracle.closest_silhouette(3, SN, SS, np.array([[1.5, 0.5, 0.5]]))
    assert r["valid"][0] and r["prim_id"][0] == 3
    assert np.allclose(r["p"][:, 0], [0.8333333, 0.1666667, 0.3333333], rtol=1e-5)
    assert math.isclose(r["d"][0], 0.7637626, rel_tol=2e-6)
    # the README tetrahedron is inconsistently oriented: edge (0,1) keeps a zero 4th vertex
    raw = gx.build_flat_silhouette_edges(TETRA_V, TETRA_F).reshape(-1, 19)
    assert np.all(raw[0, 9:12] == 0)


@pytest.mark.parametrize("seed", [0, 1])
def test_oracle_cp3d_matches_fp64_brute_force(seed):
    v, f = W.icosphere(3, amplitude=0.3, seed=seed)
    b = gx.BVH3D(v, f)
    q = W.uniform_points(3000, 3, seed=seed + 10)
    r = oracle.closest_point(3, b.node_data(), b.primitive_data(), q)
    d64, id64 = oracle.brute_closest_point(3, v, f, q)
    assert r["valid"].all()
    # FP32 error is absolute, about one ulp of the coordinates (|x| <= 2): the chosen
    # primitive is optimal up to that; different ids are ties at shared vertices/edges.
    assert np.abs(r["d"] - d64).max() < ABS_TOL


def test_oracle_cp2d_matches_fp64_brute_force():
    v, e = W.star_polyline(1000, seed=3)
    b = gx.BVH(v, e)
    q = W.uniform_points(5000, 2, seed=9)
    r = oracle.closest_point(2, b.node_data(), b.primitive_data(), q)
    d64, id64 = oracle.brute_closest_point(2, v, e, q)
    assert np.abs(r["d"] - d64).max() < ABS_TOL


def test_oracle_ray3d_matches_fp64_brute_force():
    v, f = W.icosphere(3, amplitude=0.3, seed=2)
    b = gx.BVH3D(v, f)
    o, d = W.rays(4000, 3, seed=4)
    r = oracle.intersect(3, b.node_data(), b.primitive_data(), o, d)
    t64, id64 = oracle.brute_intersect3d(v, f, o, d)
    hit64 = np.isfinite(t64)
    assert (r["valid"] == hit64).mean() > 0.999
    both = r["valid"] & hit64
    # the ray parameter error scales with the ray length (|t| <= ~4 here)
    assert (np.abs(r["d"][both] - t64[both]) / np.maximum(t64[both], 1.0)).max() < 4 * ABS_TOL


def test_ray2d_does_not_shrink_rmax_but_finds_nearest():
    # bvh.py:221/239: r_max is never shrunk in 2D; the nearest hit still wins
    v, e = W.star_polyline(1000, seed=6)
    b = gx.BVH(v, e)
    o, d = W.rays(3000, 2, seed=5)
    r = oracle.intersect(2, b.node_data(), b.primitive_data(), o, d, counts=True)
    assert r["valid"].mean() > 0.3
    assert (r["d"][r["valid"]] > 0).all()


def test_visit_counts_reported():
    v, f = W.icosphere(4, amplitude=0.15, seed=0)
    b = gx.BVH3D(v, f)
    q = W.uniform_points(500, 3, seed=3)
    r = oracle.closest_point(3, b.node_data(), b.primitive_data(), q, counts=True)
    assert (r["interior"] > 0).all() and (r["tested"] > 0).all()
