"""GPU parity: the CUDA traversals (through libgq.so) against the CPU oracle.

The exact kernels follow gQuery's visit order and must agree with the oracle bit
for bit on every record field.  The quantised 8-wide kernels must give the same
validity everywhere and the same primitive except at FP32 distance ties (distances
within 2e-6 relative).  Sizes are chosen so the oracle finishes in seconds.
"""
import math

import numpy as np
import pytest
import torch

import oracle
from gquery_b200 import _lib as L
from gquery_b200 import workloads as W
from gquery_b200.scene import Scene
from parity import REL_TOL, assert_bitwise, tie_report, to_np

pytestmark = pytest.mark.gpu

CP_FIELDS_2D = ["valid", "p", "n", "t", "d", "prim_id"]
CP_FIELDS_3D = ["valid", "p", "n", "uv", "d", "prim_id"]
RAY_FIELDS_2D = ["valid", "p", "n", "t", "d", "prim_id", "on_boundary"]
RAY_FIELDS_3D = ["valid", "p", "n", "uv", "d", "prim_id", "on_boundary"]
SIL_FIELDS = ["valid", "p", "d", "prim_id"]
ABS_TOL = 5e-7  # FP32 vs FP64 distance error: about 2 ulp of coordinates of magnitude 2


@pytest.fixture(scope="module")
def star():
    v, e = W.star_polyline(4096, seed=0)
    return Scene(v, e, 2, device=0)


@pytest.fixture(scope="module")
def mesh_c1():
    v, f = W.config1_mesh()
    return Scene(v, f, 3, device=0, build_snch=False)


@pytest.fixture(scope="module")
def mesh_c2():
    v, f = W.config2_mesh()
    return Scene(v, f, 3, device=0)


@pytest.fixture(scope="module")
def mesh_small():
    v, f = W.icosphere(4, amplitude=0.3, seed=3)
    return Scene(v, f, 3, device=0)


def _ref(scene):
    return (scene.ref_array(L.ARRAY_BVH_NODES), scene.ref_array(L.ARRAY_PRIMITIVES))


def _sref(scene):
    return (scene.ref_array(L.ARRAY_SNCH_NODES), scene.ref_array(L.ARRAY_SILHOUETTES))


# ---------------------------------------------------------------- exact, 2D

@pytest.mark.parametrize("sort", [False, True])
def test_cp2d_exact_bitwise(star, sort):
    q = W.uniform_points(65536 + 37, 2, seed=11)
    got = to_np(star.closest_point(q, variant="exact", sort=sort))
    ref = oracle.closest_point(2, *_ref(star), q)
    assert_bitwise(got, ref, CP_FIELDS_2D, "cp2d ")
    assert star.device_error() == 0


def test_ray2d_exact_bitwise(star):
    o, d = W.rays(65536, 2, seed=12)
    got = to_np(star.intersect(o, d, variant="exact", sort=True))
    ref = oracle.intersect(2, *_ref(star), o, d)
    assert_bitwise(got, ref, RAY_FIELDS_2D, "ray2d ")
    assert 0.2 < got["valid"].mean() < 1.0


def test_ray2d_exact_finite_rmax(star):
    o, d = W.rays(8192, 2, seed=13)
    rmax = np.random.default_rng(5).uniform(0.0, 2.0, size=o.shape[0]).astype(np.float32)
    got = to_np(star.intersect(o, d, torch.as_tensor(rmax), variant="exact"))
    ref = oracle.intersect(2, *_ref(star), o, d, rmax)
    assert_bitwise(got, ref, RAY_FIELDS_2D, "ray2d rmax ")


def test_sil2d_exact_bitwise(star):
    x = W.uniform_points(32768, 2, seed=14)
    got = to_np(star.closest_silhouette(x, variant="exact", sort=True))
    ref = oracle.closest_silhouette(2, *_sref(star), x)
    assert_bitwise(got, ref, SIL_FIELDS, "sil2d ")


def test_sil2d_exact_finite_rmax(star):
    x = W.uniform_points(8192, 2, seed=15)
    got = to_np(star.closest_silhouette(x, 0.25, variant="exact"))
    ref = oracle.closest_silhouette(2, *_sref(star), x, 0.25)
    assert_bitwise(got, ref, SIL_FIELDS, "sil2d rmax ")
    assert 0.0 < got["valid"].mean() < 1.0


# ---------------------------------------------------------------- exact, 3D

def test_cp3d_exact_bitwise_c1(mesh_c1):
    q = W.uniform_points(16384, 3, seed=21)
    got = to_np(mesh_c1.closest_point(q, variant="exact", sort=True))
    ref = oracle.closest_point(3, *_ref(mesh_c1), q)
    assert_bitwise(got, ref, CP_FIELDS_3D, "cp3d ")


def test_ray3d_exact_bitwise_c1(mesh_c1):
    o, d = W.rays(65536, 3, seed=22)
    got = to_np(mesh_c1.intersect(o, d, variant="exact", sort=True))
    ref = oracle.intersect(3, *_ref(mesh_c1), o, d)
    assert_bitwise(got, ref, RAY_FIELDS_3D, "ray3d ")
    assert got["valid"].mean() > 0.1


def test_sil3d_exact_bitwise_c2(mesh_c2):
    x = W.uniform_points(4096, 3, seed=23)
    got = to_np(mesh_c2.closest_silhouette(x, variant="exact", sort=True))
    ref = oracle.closest_silhouette(3, *_sref(mesh_c2), x)
    assert_bitwise(got, ref, SIL_FIELDS, "sil3d ")


def test_exact_small_mesh_all_queries(mesh_small):
    q = W.uniform_points(20000, 3, seed=24)
    o, d = W.rays(20000, 3, seed=25)
    nodes, prims = _ref(mesh_small)
    assert_bitwise(to_np(mesh_small.closest_point(q, variant="exact")), oracle.closest_point(3, nodes, prims, q),
                   CP_FIELDS_3D, "cp3d small ")
    assert_bitwise(to_np(mesh_small.intersect(o, d, variant="exact")), oracle.intersect(3, nodes, prims, o, d),
                   RAY_FIELDS_3D, "ray3d small ")
    assert_bitwise(to_np(mesh_small.closest_silhouette(q, variant="exact")), oracle.closest_silhouette(3, *_sref(mesh_small), q),
                   SIL_FIELDS, "sil3d small ")


# ---------------------------------------------------------------- wide vs exact

def test_cp3d_wide_matches_exact(mesh_c1):
    q = W.uniform_points(262144, 3, seed=31)
    a = to_np(mesh_c1.closest_point(q, variant="exact", sort=True))
    b = to_np(mesh_c1.closest_point(q, variant="wide8", sort=True))
    rep = tie_report(a, b)
    assert rep["valid_mismatch"] == 0, rep
    assert rep["prim_mismatch_not_tie"] == 0, rep
    assert rep["max_rel_d"] <= REL_TOL, rep
    assert mesh_c1.device_error() == 0


def test_ray3d_wide_matches_exact(mesh_c1):
    o, d = W.rays(262144, 3, seed=32)
    a = to_np(mesh_c1.intersect(o, d, variant="exact", sort=True))
    b = to_np(mesh_c1.intersect(o, d, variant="wide8", sort=True))
    rep = tie_report(a, b)
    assert rep["valid_mismatch"] == 0, rep
    assert rep["prim_mismatch_not_tie"] == 0, rep
    assert rep["max_rel_d"] <= REL_TOL, rep


def test_2d_wide_matches_exact(star):
    q = W.uniform_points(131072, 2, seed=33)
    rep = tie_report(to_np(star.closest_point(q, variant="exact")), to_np(star.closest_point(q, variant="wide8")))
    assert rep["valid_mismatch"] == 0 and rep["prim_mismatch_not_tie"] == 0, rep
    o, d = W.rays(131072, 2, seed=34)
    rep = tie_report(to_np(star.intersect(o, d, variant="exact")), to_np(star.intersect(o, d, variant="wide8")))
    assert rep["valid_mismatch"] == 0 and rep["prim_mismatch_not_tie"] == 0, rep


# ---------------------------------------------------------------- layouts and edges

def test_soa_aos_inputs_agree(mesh_small):
    q = W.uniform_points(5000, 3, seed=41)
    aos = torch.as_tensor(q).cuda()
    soa = aos.t().contiguous()
    a = to_np(mesh_small.closest_point(aos, variant="exact"))
    b = to_np(mesh_small.closest_point(soa, variant="exact"))
    assert_bitwise(a, b, CP_FIELDS_3D, "layout ")


@pytest.mark.parametrize("n", [0, 1, 127, 128, 129])
def test_ragged_sizes(mesh_small, n):
    q = W.uniform_points(max(n, 1), 3, seed=42)[:n]
    got = to_np(mesh_small.closest_point(torch.as_tensor(q).reshape(n, 3), variant="wide8"))
    if n:
        ref = oracle.closest_point(3, *_ref(mesh_small), q)
        rep = tie_report(got, ref)
        assert rep["valid_mismatch"] == 0 and rep["prim_mismatch_not_tie"] == 0, rep
    else:
        assert got["d"].shape == (0,)


def test_queries_on_vertices_and_far_away(mesh_small):
    v = mesh_small.vertices_host[:2000]
    far = np.full((16, 3), 1e6, np.float32)
    q = np.concatenate([v, far], axis=0)
    nodes, prims = _ref(mesh_small)
    assert_bitwise(to_np(mesh_small.closest_point(q, variant="exact")), oracle.closest_point(3, nodes, prims, q),
                   CP_FIELDS_3D, "vertices ")
    got = to_np(mesh_small.closest_point(q, variant="exact"))
    assert (got["d"][:2000] == 0).all()


def test_degenerate_scene_single_leaf():
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], np.float32)
    f = np.array([[0, 1, 2], [0, 1, 3], [1, 2, 3], [0, 2, 3]], np.int32)
    s = Scene(v, f, 3, device=0)
    q = W.uniform_points(1000, 3, seed=43)
    nodes, prims = _ref(s)
    ref = oracle.closest_point(3, nodes, prims, q)
    assert_bitwise(to_np(s.closest_point(q, variant="exact")), ref, CP_FIELDS_3D, "tetra exact ")
    rep = tie_report(to_np(s.closest_point(q, variant="wide8")), ref)
    assert rep["valid_mismatch"] == 0 and rep["prim_mismatch_not_tie"] == 0, rep


# ---------------------------------------------------------------- brute force and FP64

def test_brute_force_fp32_matches_fp64(mesh_small, star):
    q = W.uniform_points(4096, 3, seed=51)
    got = to_np(mesh_small.closest_point_brute(q))
    d64, id64 = oracle.brute_closest_point(3, mesh_small.vertices_host, mesh_small.indices_host, q)
    assert np.abs(got["d"] - d64).max() <= ABS_TOL
    q2 = W.uniform_points(4096, 2, seed=52)
    got2 = to_np(star.closest_point_brute(q2))
    d2, id2 = oracle.brute_closest_point(2, star.vertices_host, star.indices_host, q2)
    assert np.abs(got2["d"] - d2).max() <= ABS_TOL


def test_brute_f64_gpu_matches_cpu(mesh_small):
    q = W.uniform_points(2048, 3, seed=53)
    d_gpu, id_gpu = mesh_small.brute_f64("cp", q)
    d_cpu, id_cpu = oracle.brute_closest_point(3, mesh_small.vertices_host, mesh_small.indices_host, q)
    assert np.allclose(d_gpu.cpu().numpy(), d_cpu, rtol=1e-12, atol=0)
    o, d = W.rays(2048, 3, seed=54)
    t_gpu, _ = mesh_small.brute_f64("ray", o, d)
    t_cpu, _ = oracle.brute_intersect3d(mesh_small.vertices_host, mesh_small.indices_host, o, d)
    t_gpu = t_gpu.cpu().numpy()
    assert np.array_equal(np.isinf(t_gpu), np.isinf(t_cpu))
    fin = np.isfinite(t_cpu)
    assert np.allclose(t_gpu[fin], t_cpu[fin], rtol=1e-12)


def test_exact_error_vs_fp64_c1_subset(mesh_c1):
    q = W.uniform_points(8192, 3, seed=55)
    got = to_np(mesh_c1.closest_point(q, variant="exact"))
    d64, _ = mesh_c1.brute_f64("cp", q)
    d64 = d64.cpu().numpy()
    err = np.abs(got["d"].astype(np.float64) - d64)
    assert err.max() <= ABS_TOL, err.max()


# ---------------------------------------------------------------- fast variants vs exact

@pytest.mark.parametrize("variant,tuning", [
    ("coherent", None),
    ("wide8", dict(packet=1, sorted=1)),
    ("wide8", dict(packet=1, sorted=0)),
    ("wide8", dict(packet=0, persist=1, budget=16)),
    ("wide8", dict(packet=0, persist=0)),
])
def test_cp3d_fast_variants_match_exact(mesh_c1, variant, tuning):
    q = W.uniform_points(131072 + 5, 3, seed=61)
    a = to_np(mesh_c1.closest_point(q, variant="exact", sort=True))
    saved = mesh_c1.get_tuning("cp")
    try:
        if tuning is not None:
            mesh_c1.set_tuning("cp", variant, **tuning)
        b = to_np(mesh_c1.closest_point(q, variant=variant, sort=True))
    finally:
        mesh_c1.set_tuning("cp", **saved)
    rep = tie_report(a, b)
    assert rep["valid_mismatch"] == 0 and rep["prim_mismatch_not_tie"] == 0, rep
    assert rep["max_rel_d"] <= REL_TOL, rep
    assert mesh_c1.device_error() == 0


def test_auto_uses_tuning_table(mesh_small):
    q = W.uniform_points(10000, 3, seed=62)
    ref = to_np(mesh_small.closest_point(q, variant="exact"))
    for variant in ("exact", "coherent", "wide8"):
        mesh_small.set_tuning("cp", variant, packet=1)
        assert mesh_small.get_tuning("cp")["variant"] == variant
        rep = tie_report(ref, to_np(mesh_small.closest_point(q, variant="auto")))
        assert rep["valid_mismatch"] == 0 and rep["prim_mismatch_not_tie"] == 0, rep


def test_unsorted_queries_give_same_answers(mesh_c1):
    q = W.uniform_points(50000, 3, seed=63)
    a = to_np(mesh_c1.closest_point(q, variant="coherent", sort=False))
    b = to_np(mesh_c1.closest_point(q, variant="coherent", sort=True))
    rep = tie_report(a, b)
    assert rep["valid_mismatch"] == 0 and rep["prim_mismatch_not_tie"] == 0, rep


# ---------------------------------------------------------------- silhouettes: refill and coherent

@pytest.mark.parametrize("dim", [2, 3])
def test_sil_refill_bitwise_and_coherent_ties(dim, star, mesh_c2):
    scene = star if dim == 2 else mesh_c2
    n = 40000 + 17 if dim == 2 else 12000 + 3
    x = W.uniform_points(n, dim, seed=70 + dim)
    saved = scene.get_tuning("sil")
    try:
        scene.set_tuning("sil", "exact", persist=0)
        a = to_np(scene.closest_silhouette(x, variant="exact"))
        scene.set_tuning("sil", "exact", persist=1, budget=7)
        b = to_np(scene.closest_silhouette(x, variant="exact"))
    finally:
        scene.set_tuning("sil", **saved)
    assert_bitwise(b, a, SIL_FIELDS, "sil refill ")
    for r_max in (math.inf, 0.3):
        ref = to_np(scene.closest_silhouette(x, r_max, variant="exact"))
        for variant in ("coherent", "warp"):
            got = to_np(scene.closest_silhouette(x, r_max, variant=variant))
            rep = tie_report(ref, got)
            assert rep["valid_mismatch"] == 0 and rep["prim_mismatch_not_tie"] == 0, (variant, r_max, rep)
            assert rep["max_rel_d"] <= REL_TOL, (variant, r_max, rep)
    assert scene.device_error() == 0


@pytest.mark.parametrize("variant", ["coherent", "warp"])
def test_sil3d_fast_variants_against_oracle_small(mesh_small, variant):
    x = W.uniform_points(3000, 3, seed=75)
    got = to_np(mesh_small.closest_silhouette(x, variant=variant))
    ref = oracle.closest_silhouette(3, *_sref(mesh_small), x)
    rep = tie_report(ref, got)
    assert rep["valid_mismatch"] == 0 and rep["prim_mismatch_not_tie"] == 0, rep
    with pytest.raises(L.GQError, match="exact, coherent or warp"):
        mesh_small.closest_silhouette(x, variant="wide8")


@pytest.mark.parametrize("variant,tuning", [("coherent", dict(stack=0)), ("wide8", dict(packet=1, sorted=0)),
                                            ("wide8", dict(packet=1, sorted=1))])
def test_compact_stack_same_answers(mesh_c1, variant, tuning):
    """The warp-coherent walks with the compact stack (keys rounded down to FP16, one node
    word per warp).  A key rounded down only admits entries whose triangles are all
    farther than the lane's radius, so no lane's best changes: the binary walk gives the
    same records bit for bit.  In the 8-wide walk an extra lane that enters a node also
    takes part in choosing the order of its children, so a query may end on the other
    triangle of an exact distance tie: validity and distances bit for bit, primitives up
    to exact ties."""
    q = torch.as_tensor(W.uniform_points(200_000, 3, seed=57)).cuda()
    try:
        mesh_c1.set_tuning("cp", variant, **tuning)
        plain = to_np(mesh_c1.closest_point(q, variant=variant))
        mesh_c1.set_tuning("cp", variant, **dict(tuning, packet=2))
        compact = to_np(mesh_c1.closest_point(q, variant=variant))
    finally:
        mesh_c1.set_tuning("cp", "coherent", packet=1, persist=0)
    if variant == "coherent":
        assert_bitwise(compact, plain, CP_FIELDS_3D, "coherent compact ")
    else:
        assert_bitwise(compact, plain, ["valid", "d"], f"{variant} compact ")
        rep = tie_report(compact, plain)
        assert rep["prim_mismatch"] == rep["prim_mismatch_exact_tie"], rep
    assert mesh_c1.device_error() == 0


def test_ray_group_matches_exact(mesh_c1, star):
    """Rays over the 8-wide nodes with one ray per group of 8 lanes against the exact
    traversal: the same hits, the same primitive except at FP32 distance ties, and
    against the per-lane 8-wide traversal."""
    for scene, dim, fields, n in ((mesh_c1, 3, RAY_FIELDS_3D, 262_144), (star, 2, RAY_FIELDS_2D, 65_536)):
        o, d = W.rays(n, dim, seed=58 + dim)
        rm = torch.as_tensor(np.random.default_rng(59).uniform(0.2, 3.0, n).astype(np.float32))
        for r_max in (math.inf, rm):
            exact = to_np(scene.intersect(o, d, r_max, variant="exact"))
            try:
                scene.set_tuning("ray", "wide8", packet=1)
                group = to_np(scene.intersect(o, d, r_max, variant="wide8"))
                scene.set_tuning("ray", "wide8", packet=0)
                lane = to_np(scene.intersect(o, d, r_max, variant="wide8"))
            finally:
                scene.set_tuning("ray", "wide8", packet=0)
            for other, what in ((exact, "exact"), (lane, "per-lane wide8")):
                rep = tie_report(group, other)
                assert rep["valid_mismatch"] == 0 and rep["prim_mismatch_not_tie"] == 0, (dim, what, rep)
                assert rep["max_rel_d"] <= REL_TOL, (dim, what, rep)
            same = group["prim_id"] == exact["prim_id"]
            assert_bitwise({k: np.asarray(v)[..., same] for k, v in group.items()},
                           {k: np.asarray(v)[..., same] for k, v in exact.items()}, fields, f"{dim}D group ")
            assert group["valid"].any()
        assert scene.device_error() == 0


@pytest.fixture(scope="module")
def mesh_c1_16():
    v, f = W.config1_mesh()
    return Scene(v, f, 3, device=0, build_snch=False, build_wide=2)


def test_wide16_matches_exact(mesh_c1_16, star):
    """Closest points and rays over the 8-wide nodes with 16-bit child bounds against the
    exact traversal: the same validity everywhere, the same primitive except at FP32
    distance ties, distances within 2e-6 relative; and the same answers as the 8-bit
    bounds up to ties."""
    v, e = W.star_polyline(4096, seed=0)
    star16 = Scene(v, e, 2, device=0, build_snch=False, build_wide=2)
    for scene, dim, n in ((mesh_c1_16, 3, 200_000), (star16, 2, 100_000)):
        q = torch.as_tensor(W.uniform_points(n, dim, seed=60 + dim)).cuda()
        o, d = W.rays(n, dim, seed=62 + dim)
        ex_cp = to_np(scene.closest_point(q, variant="exact"))
        w16_cp = to_np(scene.closest_point(q, variant="wide16"))
        ex_ray = to_np(scene.intersect(o, d, variant="exact"))
        w16_ray = to_np(scene.intersect(o, d, variant="wide16"))
        for a, b, what in ((w16_cp, ex_cp, "cp"), (w16_ray, ex_ray, "ray")):
            rep = tie_report(a, b)
            assert rep["valid_mismatch"] == 0 and rep["prim_mismatch_not_tie"] == 0, (dim, what, rep)
            assert rep["max_rel_d"] <= REL_TOL, (dim, what, rep)
        scene.set_tuning("cp", "wide8", packet=0, persist=1)
        w8_cp = to_np(scene.closest_point(q, variant="wide8"))
        scene.set_tuning("cp", "coherent", packet=1, persist=0)
        rep = tie_report(w16_cp, w8_cp)
        assert rep["valid_mismatch"] == 0 and rep["prim_mismatch_not_tie"] == 0, (dim, rep)
        assert scene.device_error() == 0


def test_wide16_needs_the_16bit_build(mesh_c1):
    with pytest.raises(L.GQError) as ei:
        mesh_c1.closest_point(torch.zeros(64, 3, device="cuda"), variant="wide16")
    assert ei.value.status == L.GQ_ERR_UNSUPPORTED
