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
