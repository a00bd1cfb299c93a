"""Scenes built on the device (linear BVH, its collapse into quantised 8-wide nodes, the
SNCH): queries on them give the host-built scene's answers (same validity and
distances, same primitive except at FP32 ties) in every variant."""
import time

import numpy as np
import pytest

from gquery_b200 import _lib as L
from gquery_b200 import workloads as W
from gquery_b200.scene import Scene
from parity import REL_TOL, tie_report, to_np

pytestmark = pytest.mark.gpu


def _check(a, b, what):
    rep = tie_report(to_np(a), to_np(b))
    assert rep["valid_mismatch"] == 0 and rep["prim_mismatch_not_tie"] == 0 and rep["max_rel_d"] <= REL_TOL, (what, rep)


@pytest.mark.parametrize("dim", [2, 3])
def test_device_build_matches_host_build(dim):
    if dim == 2:
        v, f = W.star_polyline(20000, seed=2)
    else:
        v, f = W.icosphere(6, amplitude=0.2, seed=5)
    host = Scene(v, f, dim, device=0, build_snch=False)
    t0 = time.perf_counter()
    dev = Scene(v, f, dim, device=0, gpu_build=True)
    assert time.perf_counter() - t0 < 30.0
    assert dev.info["n_nodes"] == 2 * f.shape[0] - 1 and dev.info["n_wide_nodes"] > 0
    assert 1 <= dev.info["max_depth"] <= 64
    q = W.uniform_points(50000, dim, seed=3)
    o, d = W.rays(50000, dim, seed=4)
    ref_cp = host.closest_point(q, variant="exact")
    ref_ray = host.intersect(o, d, variant="exact")
    for variant in ("exact", "coherent", "wide8", "auto"):
        _check(ref_cp, dev.closest_point(q, variant=variant), f"cp {variant}")
    for variant in ("exact", "wide8"):
        _check(ref_ray, dev.intersect(o, d, variant=variant), f"ray {variant}")
    _check(host.intersect(o, d, 0.7, variant="exact"), dev.intersect(o, d, 0.7, variant="auto"), "ray r_max")
    assert dev.device_error() == 0


def test_device_build_limits_and_files(tmp_path):
    v, f = W.icosphere(3, seed=1)
    dev = Scene(v, f, 3, device=0, gpu_build=True)
    with pytest.raises(L.GQError, match="built on the device"):
        dev.ref_array(L.ARRAY_BVH_NODES)
    nowide = Scene(v, f, 3, device=0, gpu_build=True, build_wide=False)
    with pytest.raises(L.GQError, match="wide"):
        nowide.closest_point(W.uniform_points(10, 3, seed=0), variant="wide8")
    path = tmp_path / "dev.gqs"
    dev.save(path)
    back = Scene.load(path, device=0)
    q = W.uniform_points(5000, 3, seed=9)
    a, b = to_np(dev.closest_point(q, variant="exact")), to_np(back.closest_point(q, variant="exact"))
    for k in ("valid", "d", "prim_id"):
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k]))
    a, b = to_np(dev.closest_point(q, variant="wide8")), to_np(back.closest_point(q, variant="wide8"))
    for k in ("valid", "d", "prim_id"):
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k]))
    with pytest.raises(L.GQError, match="built on the device"):
        back.ref_array(L.ARRAY_PRIMITIVES)
    one = Scene(np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32), np.array([[0, 1, 2]], np.int32), 3,
                device=0, gpu_build=True)
    r = to_np(one.closest_point(np.array([[0.2, 0.2, 1.0]], np.float32), variant="exact"))
    assert r["valid"][0] and abs(float(r["d"][0]) - 1.0) < 1e-6


@pytest.mark.parametrize("level,amp", [(1, 0.0), (4, 0.3), (6, 0.15)])
def test_device_silhouette_edges_equal_host(level, amp):
    from gquery_b200.gquery_ext import build_flat_silhouette_edges, build_flat_silhouette_edges_device
    v, f = W.icosphere(level, amplitude=amp, seed=level)
    host = build_flat_silhouette_edges(v, f)
    dev = build_flat_silhouette_edges_device(v, f).cpu().numpy()
    assert host.shape == dev.shape
    assert np.array_equal(host.view(np.uint32), dev.view(np.uint32))


def test_device_silhouette_edges_open_and_bad_meshes():
    import torch
    from gquery_b200.gquery_ext import build_flat_silhouette_edges, build_flat_silhouette_edges_device
    v, f = W.icosphere(2, seed=1)
    f_open = f[: len(f) // 2]  # boundary edges and unused vertices
    assert np.array_equal(build_flat_silhouette_edges(v, f_open).view(np.uint32),
                          build_flat_silhouette_edges_device(v, f_open).cpu().numpy().view(np.uint32))
    bad = f.copy()
    bad[5, 1] = len(v) + 7
    with pytest.raises(L.GQError, match="out of range"):
        build_flat_silhouette_edges_device(v, bad)
    assert build_flat_silhouette_edges_device(v, f[:0]).numel() == 0


@pytest.mark.parametrize("open_mesh", [False, True])
def test_device_snch_matches_the_baseline(open_mesh):
    """The SNCH built on the device tree (cones from the geometry) answers silhouette
    queries like closest_silhouette_baseline, up to FP32 ties, in every variant."""
    v, f = W.icosphere(5, amplitude=0.3, seed=6)
    if open_mesh:
        f = f[v[f[:, 0], 2] > -0.4]  # boundary edges
    dev = Scene(v, f, 3, device=0, gpu_build=True)
    assert dev.info["n_silhouettes"] == 3 * f.shape[0]
    q = W.uniform_points(20000, 3, seed=7)
    for r_max in (np.inf, 0.3):
        base = dev.closest_silhouette_brute(q, r_max)
        for variant in ("exact", "coherent", "warp"):
            _check(base, dev.closest_silhouette(q, r_max, variant=variant), f"sil {variant} r_max={r_max}")
    assert dev.device_error() == 0


def test_device_snch_scene_file(tmp_path):
    v, f = W.icosphere(4, amplitude=0.2, seed=8)
    dev = Scene(v, f, 3, device=0, gpu_build=True)
    path = tmp_path / "dev_snch.gqs"
    dev.save(path)
    back = Scene.load(path, device=0)
    q = W.uniform_points(5000, 3, seed=10)
    a = to_np(dev.closest_silhouette(q, variant="exact"))
    b = to_np(back.closest_silhouette(q, variant="exact"))
    for k in ("valid", "d", "prim_id"):
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k]))
    one = Scene(np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32), np.array([[0, 1, 2]], np.int32), 3,
                device=0, gpu_build=True)
    x = np.array([[0.3, 0.3, 1.0], [2.0, 2.0, 0.0]], np.float32)
    _check(one.closest_silhouette_brute(x), one.closest_silhouette(x, variant="exact"), "single triangle")


@pytest.mark.parametrize("closed", [True, False])
def test_device_snch_polyline_matches_host(closed):
    """2D: the device SNCH (vertex records with the reference's last-writer neighbours,
    cones from the geometry) answers like the host-built SNCH, up to FP32 ties."""
    if closed:
        v, e = W.star_polyline(20000, seed=3)
    else:
        rng = np.random.default_rng(4)
        v = np.cumsum(rng.normal(0, 0.01, (5000, 2)), axis=0).astype(np.float32)
        e = np.stack([np.arange(4999), np.arange(1, 5000)], 1).astype(np.int32)  # open chain
    host = Scene(v, e, 2, device=0, build_snch=True, build_wide=False)
    dev = Scene(v, e, 2, device=0, gpu_build=True)
    assert dev.info["n_silhouettes"] == 2 * e.shape[0]
    lo, hi = v.min(0), v.max(0)
    q = (lo + (hi - lo) * np.random.default_rng(5).uniform(-0.5, 1.5, (20000, 2))).astype(np.float32)
    for r_max in (np.inf, 0.05):
        ref = host.closest_silhouette(q, r_max, variant="exact")
        for variant in ("exact", "coherent", "warp"):
            _check(ref, dev.closest_silhouette(q, r_max, variant=variant), f"sil2 {variant} r_max={r_max}")
    assert dev.device_error() == 0
