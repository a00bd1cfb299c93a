"""closest_point_baseline / intersect_baseline on the GPU (gq_closest_point_brute,
gq_intersect_brute) against the oracle's FP32 restatement of polyline.py:137-209 and
mesh.py:60-117, bit for bit on every record field: the 4,096-vertex star of the 2D
closest-point workload and a level-4 displaced icosphere, r_max infinite, one finite
radius for all rays and one per ray, and Polyline.intersect's on-boundary offset
(polyline.py:124-130) through the façade."""
import numpy as np
import pytest
import torch

import oracle
from gquery_b200 import workloads as W
from gquery_b200.scene import Scene
from gquery_b200.shapes import Mesh, Polyline
from parity import assert_bitwise, to_np

pytestmark = pytest.mark.gpu

CP = {2: ["valid", "p", "n", "t", "d", "prim_id"], 3: ["valid", "p", "n", "uv", "d", "prim_id"]}
RAY = {2: ["valid", "p", "n", "t", "d", "prim_id", "on_boundary"],
       3: ["valid", "p", "n", "uv", "d", "prim_id", "on_boundary"]}


def _shape(dim):
    if dim == 2:
        return W.star_polyline(4096, seed=0)
    return W.icosphere(4, amplitude=0.3, seed=3)


@pytest.fixture(scope="module", params=[2, 3], ids=["star4096", "icosphere4"])
def scene(request):
    dim = request.param
    v, ix = _shape(dim)
    return dim, v, ix, Scene(v, ix, dim, device=0, build_snch=False)


def test_closest_point_brute_bitwise(scene):
    dim, v, ix, s = scene
    q = W.uniform_points(3000, dim, seed=41)
    q[:8] = v[ix[:8, 0]]  # on vertices: zero distances
    got = to_np(s.closest_point_brute(q))
    ref = oracle.closest_point_baseline(dim, v, ix, q)
    assert_bitwise(got, ref, CP[dim], f"cp {dim}D ")
    assert got["valid"].all()


@pytest.mark.parametrize("r_max", ["inf", "scalar", "per_ray"])
def test_intersect_brute_bitwise(scene, r_max):
    dim, v, ix, s = scene
    o, d = W.rays(3000, dim, seed=42)
    if r_max == "inf":
        rm, rm_ref = np.inf, None
    elif r_max == "scalar":
        rm, rm_ref = 1.0, 1.0
    else:
        rm_ref = np.random.default_rng(43).uniform(0.0, 3.0, o.shape[0]).astype(np.float32)
        rm = torch.as_tensor(rm_ref)
    got = to_np(s.intersect_brute(o, d, rm))
    ref = oracle.intersect_baseline(dim, v, ix, o, d, rm_ref)
    assert_bitwise(got, ref, RAY[dim], f"ray {dim}D r_max={r_max} ")
    assert 0 < got["valid"].sum() < got["valid"].size


def test_polyline_intersect_offset_bitwise():
    v, e = _shape(2)
    pl = Polyline(torch.as_tensor(v), torch.as_tensor(e))
    # origins on the curve, normals of their segments, half flagged on the boundary
    rng = np.random.default_rng(44)
    seg = rng.integers(0, e.shape[0], 2000)
    t = rng.uniform(0, 1, 2000).astype(np.float32)
    a, b = v[e[seg, 0]], v[e[seg, 1]]
    x = (a + (b - a) * t[:, None]).astype(np.float32)
    tan = (b - a) / np.linalg.norm(b - a, axis=1, keepdims=True)
    n = np.stack([tan[:, 1], -tan[:, 0]], 1).astype(np.float32)
    onb = rng.random(2000) < 0.5
    _, dirs = W.rays(2000, 2, seed=45)
    got = to_np(pl.intersect(torch.as_tensor(x).cuda(), dirs, torch.as_tensor(n).cuda(), torch.as_tensor(onb).cuda()))
    x_off = np.where(onb[:, None], x - np.float32(1e-5) * n, x).astype(np.float32)
    ref = oracle.intersect_baseline(2, v, e, x_off, dirs)
    assert_bitwise(got, ref, RAY[2], "Polyline.intersect ")
    assert got["valid"].any()


def test_facade_baselines_equal_scene_calls():
    v, f = _shape(3)
    m = Mesh(torch.as_tensor(v), torch.as_tensor(f))
    q = torch.as_tensor(W.uniform_points(1000, 3, seed=46)).cuda()
    assert_bitwise(to_np(m.closest_point_baseline(q)), to_np(m.scene.closest_point_brute(q)), CP[3], "mesh cp ")
    o, d = W.rays(1000, 3, seed=47)
    assert_bitwise(to_np(m.intersect_baseline(o, d)), to_np(m.scene.intersect_brute(o, d)), RAY[3], "mesh ray ")
