"""Per-query r_max at its edges (0, negative, NaN, the smallest normal float, finite,
+inf) for rays and silhouettes in 2D and 3D: the exact variants match the oracle bit for
bit (the reference's comparisons turn 0, negative and NaN into misses), the others
match the exact variant up to FP32 ties."""
import math

import numpy as np
import pytest
import torch

import oracle
from gquery_b200 import _lib as L
from gquery_b200 import workloads as W
from gquery_b200.scene import Scene
from parity import REL_TOL, assert_bitwise, assert_sil_variant, tie_report, to_np

pytestmark = pytest.mark.gpu

EDGES = np.array([0.0, -1.0, np.nan, 1.17549435e-38, 0.35, math.inf], np.float32)


def _rmax(n):
    return np.resize(EDGES, n).astype(np.float32)


def _ties(a, b, what):
    rep = tie_report(a, b)
    assert rep["valid_mismatch"] == 0 and rep["prim_mismatch_not_tie"] == 0 and rep["max_rel_d"] <= REL_TOL, (what, rep)


@pytest.fixture(scope="module")
def scenes():
    v2, e2 = W.star_polyline(3000, seed=1)
    v3, f3 = W.icosphere(4, amplitude=0.25, seed=2)
    return {2: (Scene(v2, e2, 2, device=0), v2), 3: (Scene(v3, f3, 3, device=0), v3)}


@pytest.mark.parametrize("dim", [2, 3])
def test_rays_rmax_edges(dim, scenes):
    s, _ = scenes[dim]
    o, d = W.rays(6000, dim, seed=3)
    rm = _rmax(o.shape[0])
    got = to_np(s.intersect(o, d, torch.as_tensor(rm).cuda(), variant="exact"))
    ref = oracle.intersect(dim, s.ref_array(L.ARRAY_BVH_NODES), s.ref_array(L.ARRAY_PRIMITIVES), o, d, rm)
    fields = ["valid", "p", "n", "t" if dim == 2 else "uv", "d", "prim_id", "on_boundary"]
    assert_bitwise(got, ref, fields, f"ray{dim}d ")
    assert not got["valid"][np.isnan(rm) | (rm <= 0)].any()
    _ties(got, to_np(s.intersect(o, d, torch.as_tensor(rm).cuda(), variant="wide8")), f"ray{dim}d wide8")


@pytest.mark.parametrize("dim", [2, 3])
def test_silhouettes_rmax_edges(dim, scenes):
    s, _ = scenes[dim]
    x = W.uniform_points(6000, dim, seed=4)
    rm = _rmax(x.shape[0])
    got = to_np(s.closest_silhouette(x, torch.as_tensor(rm).cuda(), variant="exact"))
    ref = oracle.closest_silhouette(dim, s.ref_array(L.ARRAY_SNCH_NODES), s.ref_array(L.ARRAY_SILHOUETTES), x, rm)
    assert_bitwise(got, ref, ["valid", "p", "d", "prim_id"], f"sil{dim}d ")
    assert not got["valid"][np.isnan(rm) | (rm <= 0)].any()
    base = to_np(s.closest_silhouette_brute(x, torch.as_tensor(rm).cuda()))
    assert not base["valid"][np.isnan(rm) | (rm <= 0)].any()
    for variant in ("coherent", "warp"):
        assert_sil_variant(got, to_np(s.closest_silhouette(x, torch.as_tensor(rm).cuda(), variant=variant)), base,
                           f"sil{dim}d {variant}")


@pytest.mark.parametrize("scale,offset", [(1e3, 0.0), (1e-3, 0.0), (1.0, 500.0)])
def test_silhouettes_scaled_and_translated(scale, offset):
    """The silhouette pre-test and node bounds use margins relative to the coordinates:
    the same mesh and queries scaled or moved far from the origin give the oracle's
    answers (exact) and the exact answers up to ties (the others), or a nearer answer
    that is the brute-force nearest silhouette where the reference's cone test skips it."""
    v, f = W.icosphere(4, amplitude=0.25, seed=5)
    v = (v.astype(np.float64) * scale + offset).astype(np.float32)
    s = Scene(v, f, 3, device=0)
    x = (W.uniform_points(5000, 3, seed=6).astype(np.float64) * scale + offset).astype(np.float32)
    got = to_np(s.closest_silhouette(x, variant="exact"))
    ref = oracle.closest_silhouette(3, s.ref_array(L.ARRAY_SNCH_NODES), s.ref_array(L.ARRAY_SILHOUETTES), x)
    assert_bitwise(got, ref, ["valid", "p", "d", "prim_id"], f"sil scale={scale} offset={offset} ")
    assert got["valid"].mean() > 0.5
    base = to_np(s.closest_silhouette_brute(x))
    for variant in ("coherent", "warp"):
        assert_sil_variant(got, to_np(s.closest_silhouette(x, variant=variant)), base,
                           f"sil {variant} scale={scale} offset={offset}")
