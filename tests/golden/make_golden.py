"""Generates the golden fixtures in this directory by running gQuery's OWN traversal
code (gquery/shapes/bvh.py, bvh3d.py, snch.py, snch3d.py and the primitive views,
imported from the reference checkout) one query at a time under the scalar DrJit
stand-in of drjit_scalar.py.  The trees come from this project's builder through a
stand-in `gquery.gquery_ext` (the reference's nanobind builder needs Eigen, which is not
available).  What this pins: the traversal control flow, pruning and tie rules of the
reference, statement for statement.  What it cannot pin: DrJit's own rounding (the
stand-in applies this project's fixed rules, the same as the kernels and the oracle).

    python tests/golden/make_golden.py <gQuery checkout>      (or GQ_REFERENCE=<checkout>)

Writes golden_<case>.npz: scene, queries and the reference's record fields;
baseline_<case>.npz: the records of the reference's brute-force methods
(Polyline/Mesh closest_point_baseline and intersect_baseline, Polyline.intersect); and
deep_<case>.npz: the traversals on deep trees (scenes named by their generator in
gquery_b200.workloads and a checksum of the generated arrays); rmax_<case>.npz: rays and
silhouettes with a per-query finite r_max; degenerate_<case>.npz and open_<case>.npz: all three
traversals on degenerate and on open geometry.  --baselines-only, --deep-only,
--rmax-only, --degenerate-only and --open-only write one group alone.
"""
from __future__ import annotations

import os
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
_ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GQ_REFERENCE")
if not _ref:
    sys.exit("usage: make_golden.py <path of a gQuery checkout>  (or set GQ_REFERENCE)")
REF = Path(_ref)
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


def baseline_2d(name, v, e, q, o, d, rmax, nrm, onb):
    """The reference's Polyline brute-force methods on a Polyline whose flat vertex and
    index buffers are set as Polyline.__init__ sets them (polyline.py:20-33); the
    constructor itself is not run (it would build trees through the nanobind module)."""
    from drjit_scalar import Bool, Int
    from gquery.shapes.polyline import Polyline
    pl = object.__new__(Polyline)
    pl._vertices = Float(np.ascontiguousarray(v, np.float32).reshape(-1))
    pl._indices = Int(np.ascontiguousarray(e, np.int32).reshape(-1))
    cp = run(pl.closest_point_baseline, [(vec(p),) for p in q], ["valid", "p", "n", "t", "d", "prim_id"])
    fields = ["valid", "p", "n", "t", "d", "prim_id", "on_boundary"]
    ray = run(pl.intersect_baseline, [(vec(a), vec(b), Float(r)) for a, b, r in zip(o, d, rmax)], fields)
    off = run(pl.intersect, [(vec(a), vec(b), vec(n), Bool(bool(ob)), Float(r))
                             for a, b, n, ob, r in zip(o, d, nrm, onb, rmax)], fields)
    np.savez_compressed(HERE / f"baseline_{name}.npz", dim=2, vertices=v, indices=e, q=q, o=o, d=d, rmax=rmax,
                        n=nrm, on_boundary=onb, **{f"cp_{k}": x for k, x in cp.items()},
                        **{f"ray_{k}": x for k, x in ray.items()}, **{f"off_{k}": x for k, x in off.items()})
    print("baseline", name, "cp valid", cp["valid"].mean(), "ray valid", ray["valid"].mean())


def baseline_3d(name, v, f, q, o, d, rmax):
    """The reference's Mesh brute-force methods on a Mesh holding the vertex and index
    arrays and the face normals of Mesh.configure_normal (mesh.py:35-40), computed face by
    face with the same operations; the constructor itself is not run."""
    from drjit_scalar import Array3i
    from gquery.shapes.mesh import Mesh
    m = object.__new__(Mesh)
    m.vertices = soa(v, Array3)
    m.indices = soa(f, Array3i)
    fn = []
    for tri in f:
        a, b, c = (vec(v[k]) for k in tri)
        fn.append(dr.normalize(dr.cross(b - a, c - a)).numpy())
    m.face_normals = soa(np.stack(fn).astype(np.float32), Array3)
    cp = run(m.closest_point_baseline, [(vec(p),) for p in q], ["valid", "p", "n", "uv", "d", "prim_id"])
    ray = run(m.intersect_baseline, [(vec(a), vec(b), Float(r)) for a, b, r in zip(o, d, rmax)],
              ["valid", "p", "n", "uv", "d", "prim_id", "on_boundary"])
    np.savez_compressed(HERE / f"baseline_{name}.npz", dim=3, vertices=v, indices=f, q=q, o=o, d=d, rmax=rmax,
                        **{f"cp_{k}": x for k, x in cp.items()}, **{f"ray_{k}": x for k, x in ray.items()})
    print("baseline", name, "cp valid", cp["valid"].mean(), "ray valid", ray["valid"].mean())


def _rmax(n, seed):
    """+inf for even queries, a finite radius in [0.2, 2] for odd ones."""
    r = np.random.default_rng(seed).uniform(0.2, 2.0, n).astype(np.float32)
    r[0::2] = np.inf
    return r


def baselines():
    pv = np.array([[0.0, 0.0], [1.0, 0.0], [1.5, 1.0], [0.5, 1.5], [-0.5, 1.0]], np.float32)
    pe = np.array([[0, 1], [1, 2], [2, 3], [3, 4], [4, 0]], np.int32)
    for name, (v, e) in (("pentagon", (pv, pe)), ("star300", W.star_polyline(300, seed=7))):
        q = W.uniform_points(96, 2, seed=601)
        o, d = W.rays(96, 2, seed=602)
        rng = np.random.default_rng(603)
        ang = rng.uniform(0, 2 * np.pi, 96)
        nrm = np.stack([np.cos(ang), np.sin(ang)], 1).astype(np.float32)
        onb = rng.random(96) < 0.5
        baseline_2d(name, v, e, q, o, d, _rmax(96, 604), nrm, onb)
    tv = np.array([[0, 0, 0], [1, 0, 0], [0.5, 1, 0], [0.5, 0.5, 1]], np.float32)
    tf = np.array([[0, 1, 2], [0, 1, 3], [1, 2, 3], [0, 2, 3]], np.int32)
    for name, (v, f) in (("tetrahedron", (tv, tf)), ("icosphere2", W.icosphere(2, amplitude=0.3, seed=11))):
        q = W.uniform_points(96, 3, seed=605)
        o, d = W.rays(96, 3, seed=606)
        baseline_3d(name, v, f, q, o, d, _rmax(96, 607))


def geometry_checksum(v, ix):
    """sha256 of the float32 vertices and int32 indices (the deep fixtures store the
    generator of their scene and this checksum instead of the arrays)."""
    import hashlib
    h = hashlib.sha256(np.ascontiguousarray(v, np.float32).tobytes())
    h.update(np.ascontiguousarray(ix, np.int32).tobytes())
    return h.hexdigest()


DEEP = {  # name: (generator in gquery_b200.workloads, keyword arguments)
    "c2_icosphere7": ("config2_mesh", {}),
    "star262144": ("star_polyline", {"n": 262144, "seed": 1}),
}


def deep_cases(nq=256):
    """The reference's traversal on deep trees: the 327,680-triangle mesh of the
    silhouette workload (tree depth 25) and a 262,144-segment star (depth 29)."""
    from drjit_scalar import Array2i, Array3i
    for name, (gen, kw) in DEEP.items():
        v, ix = getattr(W, gen)(**kw)
        dim = v.shape[1]
        q = W.uniform_points(nq, dim, seed=710)
        o, d = W.rays(nq, dim, seed=711)
        rmax_sil = np.float32(np.inf) if dim == 3 else np.float32(0.5)
        if dim == 3:
            V, F = soa(v, Array3), soa(ix, Array3i)
            bvh, snch = BVH3D(V, F), SNCH3D(V, F)
            cpf, rayf = ["valid", "p", "n", "uv", "d", "prim_id"], ["valid", "p", "n", "uv", "d", "prim_id", "on_boundary"]
        else:
            V, F = soa(v, Array2), soa(ix, Array2i)
            bvh, snch = BVH(V, F), SNCH(V, F)
            cpf, rayf = ["valid", "p", "n", "t", "d", "prim_id"], ["valid", "p", "n", "t", "d", "prim_id", "on_boundary"]
        cp = run(bvh.closest_point, [(vec(p),) for p in q], cpf)
        ray = run(bvh.intersect, [(vec(a), vec(b), Float(dr.inf)) for a, b in zip(o, d)], rayf)
        sil = run(snch.closest_silhouette, [(vec(p), Float(rmax_sil)) for p in q], ["valid", "p", "d", "prim_id"])
        np.savez_compressed(HERE / f"deep_{name}.npz", dim=dim, generator=gen, params=str(sorted(kw.items())),
                            checksum=geometry_checksum(v, ix), q=q, o=o, d=d, rmax_sil=rmax_sil,
                            **{f"cp_{k}": x for k, x in cp.items()}, **{f"ray_{k}": x for k, x in ray.items()},
                            **{f"sil_{k}": x for k, x in sil.items()})
        print("deep", name, "cp valid", cp["valid"].mean(), "ray valid", ray["valid"].mean(),
              "sil valid", sil["valid"].mean())


def _rmax_ladder(n, seed):
    """Per-query radii: 0, tiny, small, medium, large and +inf in turn, every third
    query a random radius in [0.01, 1.5] instead."""
    ladder = np.float32([0.0, 1e-3, 0.05, 0.2, 0.5, 1.0, 2.0, np.inf])
    r = ladder[np.arange(n) % len(ladder)].copy()
    rnd = np.random.default_rng(seed).uniform(0.01, 1.5, n).astype(np.float32)
    r[2::3] = rnd[2::3]
    return r


def rmax_cases(nq=240):
    """The reference's rays and silhouettes with a per-query finite r_max (bvh.py:201,
    bvh3d.py:177, snch.py:107, snch3d.py:144): the radius bounds the walk from the first
    node on, and a ray hit at t >= r_max is no hit.  Queries include the scene's own
    vertices (distance 0 to the nearest primitive)."""
    from drjit_scalar import Array2i, Array3i
    cases = {"star4096": ("star_polyline", {"n": 4096, "seed": 3}),
             "icosphere3": ("icosphere", {"level": 3, "amplitude": 0.3, "seed": 5})}
    for name, (gen, kw) in cases.items():
        v, ix = getattr(W, gen)(**kw)
        dim = v.shape[1]
        q = W.uniform_points(nq, dim, seed=801)
        q[: nq // 8] = v[np.random.default_rng(802).choice(len(v), nq // 8, replace=False)]
        o, d = W.rays(nq, dim, seed=803)
        r_ray, r_sil = _rmax_ladder(nq, 804), _rmax_ladder(nq, 805)[::-1].copy()
        if dim == 3:
            V, F = soa(v, Array3), soa(ix, Array3i)
            bvh, snch = BVH3D(V, F), SNCH3D(V, F)
            rayf = ["valid", "p", "n", "uv", "d", "prim_id", "on_boundary"]
        else:
            V, F = soa(v, Array2), soa(ix, Array2i)
            bvh, snch = BVH(V, F), SNCH(V, F)
            rayf = ["valid", "p", "n", "t", "d", "prim_id", "on_boundary"]
        ray = run(bvh.intersect, [(vec(a), vec(b), Float(r)) for a, b, r in zip(o, d, r_ray)], rayf)
        sil = run(snch.closest_silhouette, [(vec(p), Float(r)) for p, r in zip(q, r_sil)],
                  ["valid", "p", "d", "prim_id"])
        np.savez_compressed(HERE / f"rmax_{name}.npz", dim=dim, vertices=v, indices=ix, q=q, o=o, d=d,
                            r_ray=r_ray, r_sil=r_sil, **{f"ray_{k}": x for k, x in ray.items()},
                            **{f"sil_{k}": x for k, x in sil.items()})
        print("rmax", name, "ray valid", ray["valid"].mean(), "sil valid", sil["valid"].mean())


def degenerate_cases(nq=320):
    """The reference's traversals on degenerate geometry: a mesh with a zero-area face
    (a repeated vertex), an edge collapsed to a point in several faces, repeated faces and
    a segment-like face; a polyline with a zero-length segment, repeated segments and a
    point segment.  A quarter of the queries sit on vertices, a quarter on the midpoints
    of vertex pairs."""
    v, f = W.icosphere(3, amplitude=0.2, seed=12)
    v, f = v.copy(), f.copy()
    f[10] = [f[10][0], f[10][0], f[10][1]]
    v[f[20][2]] = v[f[20][1]]
    f = np.concatenate([f, f[30:60], [[f[5][0], f[5][1], f[5][1]]]]).astype(np.int32)
    pv, pe = W.star_polyline(500, seed=3)
    pv = pv.copy()
    pv[7] = pv[6]
    pe = np.concatenate([pe, pe[100:140], [[3, 3]]]).astype(np.int32)
    for name, (vv, ix) in (("mesh", (v, f)), ("polyline", (pv, pe))):
        dim = vv.shape[1]
        rng = np.random.default_rng(901)
        k = nq // 4
        q = np.concatenate([vv[rng.integers(0, len(vv), k)],
                            0.5 * (vv[rng.integers(0, len(vv), k)] + vv[rng.integers(0, len(vv), k)]),
                            rng.uniform(-2, 2, (nq - 2 * k, dim))]).astype(np.float32)
        o, d = W.rays(nq, dim, seed=902)
        o[:k] = q[:k]  # rays leaving from vertices
        if dim == 3:
            from drjit_scalar import Array3i
            V, F = soa(vv, Array3), soa(ix, Array3i)
            bvh, snch = BVH3D(V, F), SNCH3D(V, F)
        else:
            from drjit_scalar import Array2i
            V, F = soa(vv, Array2), soa(ix, Array2i)
            bvh, snch = BVH(V, F), SNCH(V, F)
        uv = "uv" if dim == 3 else "t"
        cp = run(bvh.closest_point, [(vec(p),) for p in q], ["valid", "p", "n", uv, "d", "prim_id"])
        ray = run(bvh.intersect, [(vec(a), vec(b), Float(dr.inf)) for a, b in zip(o, d)],
                  ["valid", "p", "n", uv, "d", "prim_id", "on_boundary"])
        sil = run(snch.closest_silhouette, [(vec(p), Float(dr.inf)) for p in q], ["valid", "p", "d", "prim_id"])
        np.savez_compressed(HERE / f"degenerate_{name}.npz", dim=dim, vertices=vv, indices=ix, q=q, o=o, d=d,
                            **{f"cp_{k}": x for k, x in cp.items()}, **{f"ray_{k}": x for k, x in ray.items()},
                            **{f"sil_{k}": x for k, x in sil.items()})
        print("degenerate", name, "cp valid", cp["valid"].mean(), "ray valid", ray["valid"].mean(),
              "sil valid", sil["valid"].mean())


def open_cases(nq=320):
    """The reference's traversals on open geometry, whose boundary edges (3D) and chain
    ends (2D) are silhouettes from every side: a 700-vertex random-walk chain and a
    level-4 icosphere with a cap cut off.  Silhouettes within r_max = 0.6 (2D) and
    unbounded (3D)."""
    rng = np.random.default_rng(9)
    cv = np.cumsum(rng.uniform(-0.05, 0.05, (700, 2)), axis=0).astype(np.float32)
    ce = np.stack([np.arange(699), np.arange(1, 700)], 1).astype(np.int32)
    mv, mf = W.icosphere(4, amplitude=0.25, seed=4)
    mf = mf[mv[mf[:, 0], 2] > -0.3]
    for name, (vv, ix, rmax_sil) in (("chain", (cv, ce, 0.6)), ("cut_icosphere4", (mv, mf, np.inf))):
        dim = vv.shape[1]
        q = W.uniform_points(nq, dim, seed=911)
        q[: nq // 8] = vv[ix[np.random.default_rng(912).integers(0, len(ix), nq // 8), 0]]
        o, d = W.rays(nq, dim, seed=913)
        if dim == 3:
            from drjit_scalar import Array3i
            V, F = soa(vv, Array3), soa(ix, Array3i)
            bvh, snch = BVH3D(V, F), SNCH3D(V, F)
        else:
            from drjit_scalar import Array2i
            V, F = soa(vv, Array2), soa(ix, Array2i)
            bvh, snch = BVH(V, F), SNCH(V, F)
        uv = "uv" if dim == 3 else "t"
        cp = run(bvh.closest_point, [(vec(p),) for p in q], ["valid", "p", "n", uv, "d", "prim_id"])
        ray = run(bvh.intersect, [(vec(a), vec(b), Float(dr.inf)) for a, b in zip(o, d)],
                  ["valid", "p", "n", uv, "d", "prim_id", "on_boundary"])
        sil = run(snch.closest_silhouette, [(vec(p), Float(rmax_sil)) for p in q], ["valid", "p", "d", "prim_id"])
        np.savez_compressed(HERE / f"open_{name}.npz", dim=dim, vertices=vv, indices=ix, q=q, o=o, d=d,
                            rmax_sil=np.float32(rmax_sil), **{f"cp_{k}": x for k, x in cp.items()},
                            **{f"ray_{k}": x for k, x in ray.items()}, **{f"sil_{k}": x for k, x in sil.items()})
        print("open", name, "cp valid", cp["valid"].mean(), "ray valid", ray["valid"].mean(),
              "sil valid", sil["valid"].mean())


def main():
    if "--baselines-only" in sys.argv:
        baselines()
        return
    if "--open-only" in sys.argv:
        open_cases()
        return
    if "--degenerate-only" in sys.argv:
        degenerate_cases()
        return
    if "--rmax-only" in sys.argv:
        rmax_cases()
        return
    if "--deep-only" in sys.argv:
        deep_cases()
        return
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
    baselines()
    deep_cases()
    rmax_cases()
    degenerate_cases()
    open_cases()


if __name__ == "__main__":
    main()
