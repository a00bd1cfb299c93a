"""Queries with non-finite or huge coordinates, mixed with ordinary ones, through every
form of every query kind.  The reference's comparisons turn NaN into a miss (nothing
passes `<=`), and an infinite coordinate admits every box (inf <= inf) without any
primitive ever being nearer than +inf, so such queries walk the tree to its end and
miss.  Each traversal visits a tree node at most once, so the walk ends; the test checks
that every call returns, that the exact kernels still equal the oracle bit for bit, that
the other forms agree with exact on which queries hit, and that the ordinary queries in
the same launch get exactly the answers they get without the others."""
import numpy as np
import pytest
import torch

import oracle
from gquery_b200 import _lib as L
from gquery_b200 import workloads as W
from gquery_b200.scene import Scene
from parity import REL_TOL, assert_bitwise, assert_sil_variant, tie_report, to_np

pytestmark = pytest.mark.gpu

BAD = np.array([np.nan, np.inf, -np.inf, 1e30, -1e30], np.float32)
CP_FIELDS = {2: ["valid", "p", "n", "t", "d", "prim_id"], 3: ["valid", "p", "n", "uv", "d", "prim_id"]}
RAY_FIELDS = ["valid", "p", "d", "prim_id"]
SIL_FIELDS = ["valid", "p", "d", "prim_id"]


def _scene(dim):
    if dim == 3:
        v, f = W.icosphere(3, amplitude=0.2, seed=21)
    else:
        v, f = W.star_polyline(300, seed=22)
    return Scene(v, f, dim, device=0, build_snch=True, build_wide=2 if dim == 3 else True)


def _mixed(dim, n, seed):
    """n ordinary points U[-2,2]^dim with every 7th one given a non-finite or huge coordinate."""
    rng = np.random.default_rng(seed)
    good = rng.uniform(-2, 2, size=(n, dim)).astype(np.float32)
    mixed = good.copy()
    bad_rows = np.arange(0, n, 7)
    for j, i in enumerate(bad_rows):
        mixed[i, j % dim] = BAD[j % len(BAD)]
    return good, mixed, bad_rows


def _keep(rec, rows):
    return {k: np.asarray(x)[..., rows] for k, x in rec.items()}


@pytest.mark.parametrize("dim", [2, 3])
def test_nonfinite_closest_points(dim):
    s = _scene(dim)
    good, q, bad = _mixed(dim, 3000, 1)
    ok = np.setdiff1d(np.arange(len(q)), bad)
    nodes, prims = s.ref_array(L.ARRAY_BVH_NODES), s.ref_array(L.ARRAY_PRIMITIVES)
    exact = to_np(s.closest_point(q, variant="exact"))
    assert_bitwise(exact, oracle.closest_point(dim, nodes, prims, q), CP_FIELDS[dim], "exact vs oracle ")
    nonfin = ~np.all(np.isfinite(q), axis=1)
    assert not np.asarray(exact["valid"])[nonfin].any(), "a query with a non-finite coordinate hit"
    variants = ("exact", "coherent", "wide8") + (("wide16",) if dim == 3 else ())
    for variant in variants:
        for sort in (True, False):
            got = to_np(s.closest_point(q, variant=variant, sort=sort))
            alone = to_np(s.closest_point(good[ok], variant=variant, sort=sort))
            assert np.array_equal(np.asarray(got["valid"]), np.asarray(exact["valid"])), (variant, sort)
            rep = tie_report(_keep(got, ok), alone)
            assert rep["valid_mismatch"] == 0 and rep["prim_mismatch_not_tie"] == 0 and rep["max_rel_d"] <= REL_TOL, (
                variant, sort, rep)
    assert s.device_error() == 0


@pytest.mark.parametrize("dim", [2, 3])
def test_nonfinite_rays(dim):
    s = _scene(dim)
    o_good, o, bad_o = _mixed(dim, 3000, 2)
    d_good, d, bad_d = _mixed(dim, 3000, 3)
    d_good = d_good / np.linalg.norm(d_good, axis=1, keepdims=True)
    d = d.copy()
    fin = np.all(np.isfinite(d), axis=1) & (np.abs(d).max(axis=1) < 1e20)
    d[fin] = d_good[fin]
    d[1::11] = 0.0  # zero directions too
    bad = np.union1d(np.union1d(bad_o, bad_d), np.arange(1, len(o), 11))
    ok = np.setdiff1d(np.arange(len(o)), bad)
    nodes, prims = s.ref_array(L.ARRAY_BVH_NODES), s.ref_array(L.ARRAY_PRIMITIVES)
    exact = to_np(s.intersect(o, d, variant="exact"))
    assert_bitwise(exact, oracle.intersect(dim, nodes, prims, o, d), RAY_FIELDS, "exact vs oracle ")
    variants = ("exact", "wide8") + (("wide16",) if dim == 3 else ())
    for variant in variants:
        got = to_np(s.intersect(o, d, variant=variant))
        alone = to_np(s.intersect(o[ok], d[ok], variant=variant))
        assert_bitwise(_keep(got, ok), alone, RAY_FIELDS, f"{variant}: ordinary rays beside non-finite ones ")
        rep = tie_report(got, exact)
        assert rep["valid_mismatch"] == 0 and rep["prim_mismatch_not_tie"] == 0, (variant, rep)
    assert s.device_error() == 0


@pytest.mark.parametrize("dim", [2, 3])
def test_nonfinite_silhouettes(dim):
    s = _scene(dim)
    good, q, bad = _mixed(dim, 2000, 4)
    ok = np.setdiff1d(np.arange(len(q)), bad)
    exact = to_np(s.closest_silhouette(q, variant="exact"))
    ref = oracle.closest_silhouette(dim, s.ref_array(L.ARRAY_SNCH_NODES), s.ref_array(L.ARRAY_SILHOUETTES), q)
    assert_bitwise(exact, ref, SIL_FIELDS, "exact vs oracle ")
    nonfin = ~np.all(np.isfinite(q), axis=1)
    assert not np.asarray(exact["valid"])[nonfin].any(), "a query with a non-finite coordinate found a silhouette"
    for variant in ("exact", "coherent", "warp"):
        got = to_np(s.closest_silhouette(q, variant=variant))
        alone = to_np(s.closest_silhouette(good[ok], variant=variant))
        assert np.array_equal(np.asarray(got["valid"]), np.asarray(exact["valid"])), variant
        rep = tie_report(_keep(got, ok), alone)
        assert rep["valid_mismatch"] == 0 and rep["prim_mismatch_not_tie"] == 0 and rep["max_rel_d"] <= REL_TOL, (
            variant, rep)
    assert s.device_error() == 0


@pytest.mark.parametrize("forms", [("coherent", "wide8", "coherent"), ("split", "wide8", "warp"),
                                   ("exact", "exact", "split")])
def test_nonfinite_in_a_batch(forms):
    from gquery_b200.batch import SceneBatch
    scenes = [_scene(3), Scene(*W.icosphere(2, amplitude=0.1, seed=23), 3, device=0, build_snch=True)]
    n = 3000
    _, q, _ = _mixed(3, n, 5)
    _, o, _ = _mixed(3, n, 6)
    d = np.random.default_rng(7).standard_normal((n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    ids = np.random.default_rng(8).integers(0, len(scenes), n).astype(np.int32)
    nonfin = ~np.all(np.isfinite(q), axis=1)
    nonfin_o = ~np.all(np.isfinite(o), axis=1)
    qd, od, dd, idd = (torch.as_tensor(x).cuda() for x in (q, o, d, ids))
    cp_v, ray_v, sil_v = forms
    batch = SceneBatch(scenes, n, cp_variant=cp_v, ray_variant=ray_v, sil_variant=sil_v)
    res = batch.run(cp=(qd, idd), ray=(od, dd, idd), sil=(qd, idd))
    torch.cuda.synchronize()
    assert batch.device_error() == 0
    cp, ray, sil = to_np(res.cp), to_np(res.ray), to_np(res.sil)
    assert not np.asarray(cp["valid"])[nonfin].any() and not np.asarray(sil["valid"])[nonfin].any()
    assert not np.asarray(ray["valid"])[nonfin_o].any()
    # the ordinary queries against the single-scene exact calls on their own scene; the
    # fast silhouette forms may also answer nearer than the exact walk where that answer
    # is the brute-force nearest (the reference's cone test can skip the nearest
    # silhouette; sil_variant_report)
    for sid, sc in enumerate(scenes):
        sel = np.nonzero((ids == sid) & ~nonfin)[0]
        rep = tie_report(_keep(cp, sel), to_np(sc.closest_point(q[sel], variant="exact")))
        assert rep["valid_mismatch"] == 0 and rep["prim_mismatch_not_tie"] == 0 and rep["max_rel_d"] <= REL_TOL, (
            forms, "cp", sid, rep)
        ex_sil = to_np(sc.closest_silhouette(q[sel], variant="exact"))
        if sil_v == "exact":
            rep = tie_report(_keep(sil, sel), ex_sil)
            assert rep["valid_mismatch"] == 0 and rep["prim_mismatch_not_tie"] == 0 and rep["max_rel_d"] <= REL_TOL, (
                forms, "sil", sid, rep)
        else:
            assert_sil_variant(ex_sil, _keep(sil, sel), to_np(sc.closest_silhouette_brute(q[sel])),
                               (forms, "sil", sid))
        sel = np.nonzero((ids == sid) & ~nonfin_o)[0]
        rep = tie_report(_keep(ray, sel), to_np(sc.intersect(o[sel], d[sel], variant="exact")))
        assert rep["valid_mismatch"] == 0 and rep["prim_mismatch_not_tie"] == 0, (forms, "ray", sid, rep)
