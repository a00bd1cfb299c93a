"""Generates the golden fixtures in this directory by running gQuery's OWN traversal
code (gquery/shapes/bvh.py, bvh3d.py, snch.py, snch3d.py and the primitive views,
imported from the reference checkout) one query at a time under the scalar DrJit
stand-in of drjit_scalar.py.  The trees come from this project's builder through a
stand-in `gquery.gquery_ext` (the reference's nanobind builder needs Eigen, which is not
available).  What this pins: the traversal control flow, pruning and tie rules of the
reference, statement for statement.  What it cannot pin: DrJit's own rounding (the
stand-in applies this project's fixed rules, the same as the kernels and the oracle).

    python tests/golden/make_golden.py [/path/to/reference]

Writes golden_<case>.npz: scene, queries and the reference's record fields.
"""
from __future__ import annotations

import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
REF = Path(sys.argv[1]) if len(sys.argv) > 1 else Path("/root/reference")
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(HERE))

import drjit_scalar  # noqa: E402

dr = drjit_scalar.install()
from drjit_scalar import Array2, Array3, Float  # noqa: E402

from gquery_b200 import gquery_ext as builder  # noqa: E402
from gquery_b200 import workloads as W  # noqa: E402

ext = types.ModuleType("gquery.gquery_ext")
ext.BVH = builder.BVH
ext.BVH3D = builder.BVH3D
ext.SNCH = builder.SNCH
ext.SNCH3D = builder.SNCH3D
sys.modules["gquery.gquery_ext"] = ext
sys.path.insert(0, str(REF))

from gquery.shapes.bvh import BVH  # noqa: E402
from gquery.shapes.bvh3d import BVH3D  # noqa: E402
from gquery.shapes.snch import SNCH  # noqa: E402
from gquery.shapes.snch3d import SNCH3D  # noqa: E402


def vec(a):
    return Array2(Float(a[0]), Float(a[1])) if len(a) == 2 else Array3(Float(a[0]), Float(a[1]), Float(a[2]))


def soa(arr, T):
    return T(np.ascontiguousarray(arr.T))


def f32(x):
    return np.float32(x.v)


def record(rec, fields):
    out = {}
    for name in fields:
        val = getattr(rec, name)
        if hasattr(val, "c"):
            out[name] = np.array([np.asarray(x.v) for x in val.c])
        else:
            out[name] = np.asarray(val.v)
    return out


def run(fn, args_list, fields):
    rows = [record(fn(*a), fields) for a in args_list]
    return {f: np.stack([r[f] for r in rows], axis=-1) for f in fields}


def case_2d(name, v, e, q, o, d, rmax_sil):
    from drjit_scalar import Array2i
    V, E = soa(v, Array2), soa(e, Array2i)
    bvh, snch = BVH(V, E), SNCH(V, E)
    cp = run(bvh.closest_point, [(vec(p),) for p in q], ["valid", "p", "n", "t", "d", "prim_id"])
    ray = run(bvh.intersect, [(vec(a), vec(b), Float(dr.inf)) for a, b in zip(o, d)],
              ["valid", "p", "n", "t", "d", "prim_id", "on_boundary"])
    sil = run(snch.closest_silhouette, [(vec(p), Float(rmax_sil)) for p in q], ["valid", "p", "d", "prim_id"])
    np.savez_compressed(HERE / f"golden_{name}.npz", dim=2, vertices=v, indices=e, q=q, o=o, d=d,
                        rmax_sil=np.float32(rmax_sil),
                        **{f"cp_{k}": x for k, x in cp.items()}, **{f"ray_{k}": x for k, x in ray.items()},
                        **{f"sil_{k}": x for k, x in sil.items()})
    print(name, "cp valid", cp["valid"].mean(), "ray valid", ray["valid"].mean(), "sil valid", sil["valid"].mean())


def case_3d(name, v, f, q, o, d, rmax_sil):
    from drjit_scalar import Array3i
    V, F = soa(v, Array3), soa(f, Array3i)
    bvh, snch = BVH3D(V, F), SNCH3D(V, F)
    cp = run(bvh.closest_point, [(vec(p),) for p in q], ["valid", "p", "n", "uv", "d", "prim_id"])
    ray = run(bvh.intersect, [(vec(a), vec(b), Float(dr.inf)) for a, b in zip(o, d)],
              ["valid", "p", "n", "uv", "d", "prim_id", "on_boundary"])
    sil = run(snch.closest_silhouette, [(vec(p), Float(rmax_sil)) for p in q], ["valid", "p", "d", "prim_id"])
    np.savez_compressed(HERE / f"golden_{name}.npz", dim=3, vertices=v, indices=f, q=q, o=o, d=d,
                        rmax_sil=np.float32(rmax_sil),
                        **{f"cp_{k}": x for k, x in cp.items()}, **{f"ray_{k}": x for k, x in ray.items()},
                        **{f"sil_{k}": x for k, x in sil.items()})
    print(name, "cp valid", cp["valid"].mean(), "ray valid", ray["valid"].mean(), "sil valid", sil["valid"].mean())


def main():
    # README pentagon (examples/example_2d.py) and tetrahedron (examples/example_3d.py)
    pv = np.array([[0.0, 0.0], [1.0, 0.0], [1.5, 1.0], [0.5, 1.5], [-0.5, 1.0]], np.float32)
    pe = np.array([[0, 1], [1, 2], [2, 3], [3, 4], [4, 0]], np.int32)
    q = np.concatenate([np.float32([[0.8, 0.8], [2.0, 0.5]]), W.uniform_points(64, 2, seed=501)])
    o, d = W.rays(64, 2, seed=502)
    o = np.concatenate([np.float32([[0.8, 0.8]]), o])
    d = np.concatenate([np.float32([[1.0, 1.0]]), d])
    case_2d("pentagon", pv, pe, q, o, d, np.inf)

    tv = np.array([[0, 0, 0], [1, 0, 0], [0.5, 1, 0], [0.5, 0.5, 1]], np.float32)
    tf = np.array([[0, 1, 2], [0, 1, 3], [1, 2, 3], [0, 2, 3]], np.int32)
    q = np.concatenate([np.float32([[0.6, 0.6, 0.6], [1.5, 0.5, 0.5]]), W.uniform_points(64, 3, seed=503)])
    o, d = W.rays(64, 3, seed=504)
    o = np.concatenate([np.float32([[0.6, 0.6, 0.6]]), o])
    d = np.concatenate([np.float32([[1.0, 1.0, 1.0]]), d])
    case_3d("tetrahedron", tv, tf, q, o, d, np.inf)

    sv, se = W.star_polyline(300, seed=7)
    q = W.uniform_points(300, 2, seed=505)
    o, d = W.rays(300, 2, seed=506)
    case_2d("star300", sv, se, q, o, d, 0.6)

    iv, iff = W.icosphere(2, amplitude=0.3, seed=11)
    q = W.uniform_points(200, 3, seed=507)
    o, d = W.rays(300, 3, seed=508)
    case_3d("icosphere2", iv, iff, q, o, d, np.inf)


if __name__ == "__main__":
    main()
