"""closest_silhouette_baseline on the GPU (gq_closest_silhouette_brute) against the
oracle's restatement, bit for bit: closed and open polylines (endpoints without a
neighbour, a collinear vertex), closed and open meshes (boundary edges), finite and
infinite r_max, and through the Polyline / Mesh façade."""
import numpy as np
import pytest
import torch

import oracle
from gquery_b200 import _lib as L
from gquery_b200 import workloads as W
from gquery_b200.scene import Scene
from gquery_b200.shapes import Mesh, Polyline
from parity import assert_bitwise, to_np

pytestmark = pytest.mark.gpu

SIL = ["valid", "p", "d", "prim_id"]


def _polylines():
    v, e = W.star_polyline(500, seed=2)
    v = v.copy()
    v[10] = 0.5 * (v[9] + v[11])  # collinear
    rng = np.random.default_rng(3)
    ov = rng.uniform(-1, 1, (60, 2)).astype(np.float32)
    oe = np.stack([np.arange(59), np.arange(1, 60)], 1).astype(np.int32)  # open chain
    return [(v, e), (ov, oe)]


@pytest.mark.parametrize("case", [0, 1])
@pytest.mark.parametrize("r_max", [np.inf, 0.3])
def test_polyline_baseline_bitwise(case, r_max):
    v, e = _polylines()[case]
    s = Scene(v, e, 2, device=0, build_snch=False)
    x = W.uniform_points(5000, 2, seed=10 + case)
    got = to_np(s.closest_silhouette_brute(x, r_max))
    ref = oracle.closest_silhouette_brute(2, x, None if np.isinf(r_max) else r_max, vertices=v, indices=e)
    assert_bitwise(got, ref, SIL, f"polyline {case} ")
    assert got["valid"].any()


@pytest.mark.parametrize("open_mesh", [False, True])
@pytest.mark.parametrize("r_max", [np.inf, 0.4])
def test_mesh_baseline_bitwise(open_mesh, r_max):
    v, f = W.icosphere(3, amplitude=0.25, seed=4)
    if open_mesh:
        f = f[v[f[:, 0], 2] > -0.3]  # cut a cap off: boundary edges
    s = Scene(v, f, 3, device=0, build_snch=True)
    x = W.uniform_points(4000, 3, seed=20)
    got = to_np(s.closest_silhouette_brute(x, r_max))
    raw = s.ref_array(L.ARRAY_RAW_SILHOUETTES)
    ref = oracle.closest_silhouette_brute(3, x, None if np.isinf(r_max) else r_max, raw_silhouettes=raw)
    assert_bitwise(got, ref, SIL, f"mesh open={open_mesh} ")
    assert got["valid"].any()


def test_baseline_through_the_facade():
    v, f = W.icosphere(3, amplitude=0.25, seed=4)
    m = Mesh(torch.as_tensor(v), torch.as_tensor(f))
    x = torch.as_tensor(W.uniform_points(3000, 3, seed=21)).cuda()
    base = to_np(m.closest_silhouette_baseline(x))
    assert_bitwise(base, to_np(m.scene.closest_silhouette_brute(x)), SIL, "facade ")
    snch = to_np(m.closest_silhouette_snch(x))
    # the SNCH walk finds the same nearest silhouette distance for (nearly) every query;
    # its cone test takes the node radius from edge midpoints (snch.cpp:117), so an edge
    # reaching just beyond it can be pruned
    same = (base["valid"] == snch["valid"]) & (~base["valid"] | np.isclose(base["d"], snch["d"], rtol=2e-6, atol=0))
    assert same.mean() >= 0.99, same.mean()
    pv, pe = _polylines()[0]
    p = Polyline(torch.as_tensor(pv), torch.as_tensor(pe))
    assert to_np(p.closest_silhouette_baseline(torch.as_tensor(W.uniform_points(100, 2, seed=5)).cuda()))["valid"].any()
