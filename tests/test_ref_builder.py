"""The builder against gQuery's OWN builder code.

oracle/_ref/libgqref.so is compiled (oracle/Makefile, `make ref`) from the reference's
src/shapes/bvh.cpp, snch.cpp and silhouette_edge.cpp, unchanged, with its thread pool
initialised to one thread (ParallelInit(1), so the builds above 131,072 primitives run
as the reference would with a pool) and a stand-in for the few Eigen operations they
use (oracle/eigen_subset).  Every reference array this project returns
(gq_scene_ref_array: node_data, primitive_data, SNCH node_data, silhouette_data,
raw_silhouette_data; build_flat_silhouette_edges) must equal the reference's bit for bit.
"""
import numpy as np
import pytest

import oracle
from gquery_b200 import _lib as L
from gquery_b200 import gquery_ext as gx
from gquery_b200 import workloads as W
from gquery_b200.scene import Scene

if oracle.build_ref() is None:
    pytest.skip("the reference builder is not built here (no gQuery checkout)", allow_module_level=True)

ARRAYS = {"bvh_nodes": L.ARRAY_BVH_NODES, "primitives": L.ARRAY_PRIMITIVES, "snch_nodes": L.ARRAY_SNCH_NODES,
          "silhouettes": L.ARRAY_SILHOUETTES, "raw_silhouettes": L.ARRAY_RAW_SILHOUETTES}


def _open_chain():
    rng = np.random.default_rng(9)
    v = np.cumsum(rng.uniform(-0.05, 0.05, (700, 2)), axis=0).astype(np.float32)
    e = np.stack([np.arange(699), np.arange(1, 700)], 1).astype(np.int32)
    return v, e


def _open_mesh():
    v, f = W.icosphere(4, amplitude=0.25, seed=4)
    return v, f[v[f[:, 0], 2] > -0.3]  # a cap cut off: boundary edges


def _cone():
    """A closed cone whose apex (vertex 0) meets 200 edges, plus a repeated face and a
    face with a repeated vertex: the edge pass sorts a bucket this large."""
    n = 200
    a = 2 * np.pi * np.arange(n) / n
    ring = np.stack([np.cos(a), np.sin(a), np.zeros(n)], 1)
    v = np.concatenate([[[0.0, 0.0, 1.0]], ring, [[0.0, 0.0, 0.0]]]).astype(np.float32)
    i = np.arange(n)
    side = np.stack([np.zeros(n, int), 1 + i, 1 + (i + 1) % n], 1)
    base = np.stack([np.full(n, n + 1), 1 + (i + 1) % n, 1 + i], 1)
    return v, np.concatenate([side, base, side[:1], [[0, 0, 5]]]).astype(np.int32)


CASES = {
    "pentagon": lambda: (np.array([[0, 0], [1, 0], [1.5, 1], [0.5, 1.5], [-0.5, 1]], np.float32),
                         np.array([[0, 1], [1, 2], [2, 3], [3, 4], [4, 0]], np.int32)),
    "star4096": lambda: W.star_polyline(4096, seed=0),
    "open_chain": _open_chain,
    "tetrahedron": lambda: (np.array([[0, 0, 0], [1, 0, 0], [0.5, 1, 0], [0.5, 0.5, 1]], np.float32),
                            np.array([[0, 1, 2], [0, 1, 3], [1, 2, 3], [0, 2, 3]], np.int32)),
    "icosphere3": lambda: W.icosphere(3, amplitude=0.3, seed=3),
    "icosphere4_open": _open_mesh,
    "icosphere5": lambda: W.icosphere(5, amplitude=0.15, seed=1),
    "cone200": _cone,
}


def _assert_same(ref, ours, what):
    assert ref.shape == ours.shape, f"{what}: length {ref.shape} vs {ours.shape}"
    bad = ref.view(np.uint32) != ours.view(np.uint32)
    assert not bad.any(), f"{what}: {int(bad.sum())} floats differ, first at {int(np.argmax(bad))}"


@pytest.mark.parametrize("name", list(CASES))
def test_reference_arrays_bitwise(name):
    v, ix = CASES[name]()
    dim = v.shape[1]
    ref = oracle.reference_build(dim, v, ix)
    s = Scene(v, ix, dim, device=None, build_snch=True)
    for k, which in ARRAYS.items():
        _assert_same(ref[k], s.ref_array(which), f"{name} {k}")


@pytest.mark.parametrize("max_prims", [1, 4])
def test_reference_arrays_other_leaf_sizes(max_prims):
    v, f = W.icosphere(4, amplitude=0.3, seed=5)
    ref = oracle.reference_build(3, v, f, max_prims_in_node=max_prims)
    s = Scene(v, f, 3, device=None, build_snch=True, max_prims_in_node=max_prims)
    for k, which in ARRAYS.items():
        _assert_same(ref[k], s.ref_array(which), f"max_prims={max_prims} {k}")


def test_flat_silhouette_edges_bitwise():
    for v, f in (W.icosphere(4, amplitude=0.3, seed=3), _open_mesh(), _cone()):
        _assert_same(oracle.reference_flat_silhouette_edges(v, f), gx.build_flat_silhouette_edges(v, f), "edges")


def test_reference_arrays_above_the_thread_pool_threshold():
    # 327,680 triangles: the reference's recursion hands its two halves to ParallelFor
    # above 131,072 primitives (bvh.cpp:281-292); with a one-thread pool it builds the
    # left half first, as this project's deterministic build does
    v, f = W.config2_mesh()
    ref = oracle.reference_build(3, v, f, snch=False)
    s = Scene(v, f, 3, device=None, build_snch=False, build_wide=False)
    for k in ("bvh_nodes", "primitives"):
        _assert_same(ref[k], s.ref_array(ARRAYS[k]), f"level 7 {k}")
