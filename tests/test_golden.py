"""Golden fixtures from gQuery's own traversal code (tests/golden/make_golden.py runs the
reference's bvh.py / bvh3d.py / snch.py / snch3d.py under a scalar DrJit stand-in).

CPU: the oracle must reproduce every record field bit for bit.  GPU: so must the exact
kernels through the C ABI."""
from pathlib import Path

import numpy as np
import pytest

import oracle
from gquery_b200 import _lib as L
from gquery_b200.scene import Scene
from parity import assert_bitwise, to_np

GOLDEN = sorted((Path(__file__).resolve().parent / "golden").glob("golden_*.npz"))
CP = {2: ["valid", "p", "n", "t", "d", "prim_id"], 3: ["valid", "p", "n", "uv", "d", "prim_id"]}
RAY = {2: ["valid", "p", "n", "t", "d", "prim_id", "on_boundary"],
       3: ["valid", "p", "n", "uv", "d", "prim_id", "on_boundary"]}
SIL = ["valid", "p", "d", "prim_id"]


def load(path):
    z = np.load(path)
    dim = int(z["dim"])
    return dim, z


def expected(z, prefix, fields):
    return {f: z[f"{prefix}_{f}"] for f in fields}


def test_fixtures_exist():
    names = {p.stem for p in GOLDEN}
    assert {"golden_pentagon", "golden_tetrahedron", "golden_star300", "golden_icosphere2"} <= names


@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_oracle_matches_reference_traversal(path):
    dim, z = load(path)
    s = Scene(z["vertices"], z["indices"], dim, device=None)
    nodes, prims = s.ref_array(L.ARRAY_BVH_NODES), s.ref_array(L.ARRAY_PRIMITIVES)
    snodes, sils = s.ref_array(L.ARRAY_SNCH_NODES), s.ref_array(L.ARRAY_SILHOUETTES)
    rmax = float(z["rmax_sil"])
    assert_bitwise(oracle.closest_point(dim, nodes, prims, z["q"]), expected(z, "cp", CP[dim]), CP[dim], "cp ")
    assert_bitwise(oracle.intersect(dim, nodes, prims, z["o"], z["d"]), expected(z, "ray", RAY[dim]), RAY[dim],
                   "ray ")
    got = oracle.closest_silhouette(dim, snodes, sils, z["q"], None if np.isinf(rmax) else rmax)
    assert_bitwise(got, expected(z, "sil", SIL), SIL, "sil ")


@pytest.mark.gpu
@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_exact_kernels_match_reference_traversal(path):
    dim, z = load(path)
    s = Scene(z["vertices"], z["indices"], dim, device=0)
    rmax = float(z["rmax_sil"])
    assert_bitwise(to_np(s.closest_point(z["q"], variant="exact")), expected(z, "cp", CP[dim]), CP[dim], "cp ")
    assert_bitwise(to_np(s.intersect(z["o"], z["d"], variant="exact")), expected(z, "ray", RAY[dim]), RAY[dim],
                   "ray ")
    assert_bitwise(to_np(s.closest_silhouette(z["q"], rmax, variant="exact")), expected(z, "sil", SIL), SIL, "sil ")


# ---------------------------------------------------------------- brute-force baselines

BASELINES = sorted((Path(__file__).resolve().parent / "golden").glob("baseline_*.npz"))


def _offset(z):
    """Polyline.intersect's origin (polyline.py:124-130): x - 1e-5 n where on_boundary."""
    return np.where(z["on_boundary"][:, None], z["o"] - np.float32(1e-5) * z["n"], z["o"]).astype(np.float32)


def test_baseline_fixtures_exist():
    names = {p.stem for p in BASELINES}
    assert {"baseline_pentagon", "baseline_star300", "baseline_tetrahedron", "baseline_icosphere2"} <= names


@pytest.mark.parametrize("path", BASELINES, ids=[p.stem for p in BASELINES])
def test_oracle_matches_reference_baselines(path):
    dim, z = load(path)
    v, ix = z["vertices"], z["indices"]
    assert_bitwise(oracle.closest_point_baseline(dim, v, ix, z["q"]), expected(z, "cp", CP[dim]), CP[dim], "cp ")
    assert_bitwise(oracle.intersect_baseline(dim, v, ix, z["o"], z["d"], z["rmax"]), expected(z, "ray", RAY[dim]),
                   RAY[dim], "ray ")
    if dim == 2:
        assert_bitwise(oracle.intersect_baseline(dim, v, ix, _offset(z), z["d"], z["rmax"]),
                       expected(z, "off", RAY[dim]), RAY[dim], "offset ray ")


@pytest.mark.gpu
@pytest.mark.parametrize("path", BASELINES, ids=[p.stem for p in BASELINES])
def test_brute_kernels_match_reference_baselines(path):
    import torch
    from gquery_b200.shapes import Mesh, Polyline
    dim, z = load(path)
    s = Scene(z["vertices"], z["indices"], dim, device=0, build_snch=False)
    assert_bitwise(to_np(s.closest_point_brute(z["q"])), expected(z, "cp", CP[dim]), CP[dim], "cp ")
    assert_bitwise(to_np(s.intersect_brute(z["o"], z["d"], torch.as_tensor(z["rmax"]))), expected(z, "ray", RAY[dim]),
                   RAY[dim], "ray ")
    shape = (Polyline if dim == 2 else Mesh)(torch.as_tensor(z["vertices"]), torch.as_tensor(z["indices"]))
    assert_bitwise(to_np(shape.closest_point_baseline(torch.as_tensor(z["q"]).cuda())), expected(z, "cp", CP[dim]),
                   CP[dim], "facade cp ")
    assert_bitwise(to_np(shape.intersect_baseline(z["o"], z["d"], torch.as_tensor(z["rmax"]))),
                   expected(z, "ray", RAY[dim]), RAY[dim], "facade ray ")
    if dim == 2:
        got = shape.intersect(torch.as_tensor(z["o"]).cuda(), z["d"], torch.as_tensor(z["n"]).cuda(),
                              torch.as_tensor(z["on_boundary"]).cuda(), torch.as_tensor(z["rmax"]))
        assert_bitwise(to_np(got), expected(z, "off", RAY[dim]), RAY[dim], "Polyline.intersect ")


# ---------------------------------------------------------------- deep trees

DEEP = sorted((Path(__file__).resolve().parent / "golden").glob("deep_*.npz"))


def _deep_scene(z, device):
    """The fixture's scene, regenerated by its generator; skipped when the regenerated
    arrays do not match the checksum recorded with the fixture."""
    import ast
    import hashlib
    from gquery_b200 import workloads as W
    v, ix = getattr(W, str(z["generator"]))(**dict(ast.literal_eval(str(z["params"]))))
    h = hashlib.sha256(np.ascontiguousarray(v, np.float32).tobytes())
    h.update(np.ascontiguousarray(ix, np.int32).tobytes())
    if h.hexdigest() != str(z["checksum"]):
        pytest.skip("the scene generator does not reproduce the fixture's geometry on this machine")
    return Scene(v, ix, int(z["dim"]), device=device)


def test_deep_fixtures_exist():
    assert {"deep_c2_icosphere7", "deep_star262144"} <= {p.stem for p in DEEP}


@pytest.mark.parametrize("path", DEEP, ids=[p.stem for p in DEEP])
def test_oracle_matches_reference_traversal_deep(path):
    dim, z = load(path)
    s = _deep_scene(z, None)
    nodes, prims = s.ref_array(L.ARRAY_BVH_NODES), s.ref_array(L.ARRAY_PRIMITIVES)
    snodes, sils = s.ref_array(L.ARRAY_SNCH_NODES), s.ref_array(L.ARRAY_SILHOUETTES)
    rmax = float(z["rmax_sil"])
    assert_bitwise(oracle.closest_point(dim, nodes, prims, z["q"]), expected(z, "cp", CP[dim]), CP[dim], "cp ")
    assert_bitwise(oracle.intersect(dim, nodes, prims, z["o"], z["d"]), expected(z, "ray", RAY[dim]), RAY[dim],
                   "ray ")
    got = oracle.closest_silhouette(dim, snodes, sils, z["q"], None if np.isinf(rmax) else rmax)
    assert_bitwise(got, expected(z, "sil", SIL), SIL, "sil ")


@pytest.mark.gpu
@pytest.mark.parametrize("path", DEEP, ids=[p.stem for p in DEEP])
def test_exact_kernels_match_reference_traversal_deep(path):
    dim, z = load(path)
    s = _deep_scene(z, 0)
    rmax = float(z["rmax_sil"])
    assert_bitwise(to_np(s.closest_point(z["q"], variant="exact")), expected(z, "cp", CP[dim]), CP[dim], "cp ")
    assert_bitwise(to_np(s.intersect(z["o"], z["d"], variant="exact")), expected(z, "ray", RAY[dim]), RAY[dim],
                   "ray ")
    assert_bitwise(to_np(s.closest_silhouette(z["q"], rmax, variant="exact")), expected(z, "sil", SIL), SIL, "sil ")


# ---------------------------------------------------------------- per-query finite r_max

RMAX = sorted((Path(__file__).resolve().parent / "golden").glob("rmax_*.npz"))


def test_rmax_fixtures_exist():
    assert {"rmax_star4096", "rmax_icosphere3"} <= {p.stem for p in RMAX}


@pytest.mark.parametrize("path", RMAX, ids=[p.stem for p in RMAX])
def test_oracle_matches_reference_traversal_rmax(path):
    """Rays and silhouettes with one radius per query (0, tiny, finite, +inf): the
    reference's records from bvh.py:201 / bvh3d.py:177 / snch.py:107 / snch3d.py:144."""
    dim, z = load(path)
    s = Scene(z["vertices"], z["indices"], dim, device=None)
    nodes, prims = s.ref_array(L.ARRAY_BVH_NODES), s.ref_array(L.ARRAY_PRIMITIVES)
    snodes, sils = s.ref_array(L.ARRAY_SNCH_NODES), s.ref_array(L.ARRAY_SILHOUETTES)
    assert_bitwise(oracle.intersect(dim, nodes, prims, z["o"], z["d"], z["r_ray"]), expected(z, "ray", RAY[dim]),
                   RAY[dim], "ray ")
    assert_bitwise(oracle.closest_silhouette(dim, snodes, sils, z["q"], z["r_sil"]), expected(z, "sil", SIL), SIL,
                   "sil ")


@pytest.mark.gpu
@pytest.mark.parametrize("path", RMAX, ids=[p.stem for p in RMAX])
def test_exact_kernels_match_reference_traversal_rmax(path):
    dim, z = load(path)
    s = Scene(z["vertices"], z["indices"], dim, device=0)
    assert_bitwise(to_np(s.intersect(z["o"], z["d"], z["r_ray"], variant="exact")), expected(z, "ray", RAY[dim]),
                   RAY[dim], "ray ")
    assert_bitwise(to_np(s.closest_silhouette(z["q"], z["r_sil"], variant="exact")), expected(z, "sil", SIL), SIL,
                   "sil ")
    assert s.device_error() == 0


# ---------------------------------------------------------------- degenerate geometry

DEGENERATE = sorted((Path(__file__).resolve().parent / "golden").glob("degenerate_*.npz"))


def test_degenerate_fixtures_exist():
    assert {"degenerate_mesh", "degenerate_polyline"} <= {p.stem for p in DEGENERATE}


@pytest.mark.parametrize("path", DEGENERATE, ids=[p.stem for p in DEGENERATE])
def test_oracle_matches_reference_traversal_degenerate(path):
    """Zero-area and segment-like faces, collapsed edges, repeated primitives, point
    segments; queries and ray origins on vertices: every record field of the reference."""
    dim, z = load(path)
    s = Scene(z["vertices"], z["indices"], dim, device=None)
    nodes, prims = s.ref_array(L.ARRAY_BVH_NODES), s.ref_array(L.ARRAY_PRIMITIVES)
    snodes, sils = s.ref_array(L.ARRAY_SNCH_NODES), s.ref_array(L.ARRAY_SILHOUETTES)
    assert_bitwise(oracle.closest_point(dim, nodes, prims, z["q"]), expected(z, "cp", CP[dim]), CP[dim], "cp ")
    assert_bitwise(oracle.intersect(dim, nodes, prims, z["o"], z["d"]), expected(z, "ray", RAY[dim]), RAY[dim],
                   "ray ")
    assert_bitwise(oracle.closest_silhouette(dim, snodes, sils, z["q"]), expected(z, "sil", SIL), SIL, "sil ")


@pytest.mark.gpu
@pytest.mark.parametrize("path", DEGENERATE, ids=[p.stem for p in DEGENERATE])
def test_exact_kernels_match_reference_traversal_degenerate(path):
    dim, z = load(path)
    s = Scene(z["vertices"], z["indices"], dim, device=0)
    assert_bitwise(to_np(s.closest_point(z["q"], variant="exact")), expected(z, "cp", CP[dim]), CP[dim], "cp ")
    assert_bitwise(to_np(s.intersect(z["o"], z["d"], variant="exact")), expected(z, "ray", RAY[dim]), RAY[dim],
                   "ray ")
    assert_bitwise(to_np(s.closest_silhouette(z["q"], variant="exact")), expected(z, "sil", SIL), SIL, "sil ")
    assert s.device_error() == 0


# ---------------------------------------------------------------- open geometry

OPEN = sorted((Path(__file__).resolve().parent / "golden").glob("open_*.npz"))


def test_open_fixtures_exist():
    assert {"open_chain", "open_cut_icosphere4"} <= {p.stem for p in OPEN}


@pytest.mark.parametrize("path", OPEN, ids=[p.stem for p in OPEN])
def test_oracle_matches_reference_traversal_open(path):
    """An open chain (its two ends are silhouettes from every side) and a mesh with a cap
    cut off (its boundary edges are silhouettes from every side)."""
    dim, z = load(path)
    s = Scene(z["vertices"], z["indices"], dim, device=None)
    nodes, prims = s.ref_array(L.ARRAY_BVH_NODES), s.ref_array(L.ARRAY_PRIMITIVES)
    snodes, sils = s.ref_array(L.ARRAY_SNCH_NODES), s.ref_array(L.ARRAY_SILHOUETTES)
    rmax = float(z["rmax_sil"])
    assert_bitwise(oracle.closest_point(dim, nodes, prims, z["q"]), expected(z, "cp", CP[dim]), CP[dim], "cp ")
    assert_bitwise(oracle.intersect(dim, nodes, prims, z["o"], z["d"]), expected(z, "ray", RAY[dim]), RAY[dim],
                   "ray ")
    got = oracle.closest_silhouette(dim, snodes, sils, z["q"], None if np.isinf(rmax) else rmax)
    assert_bitwise(got, expected(z, "sil", SIL), SIL, "sil ")
