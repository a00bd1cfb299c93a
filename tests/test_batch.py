"""Batched queries over many uneven scenes in one launch (gq_batch_*).

Every query must get the answer it gets from the single-scene call on its own scene:
rays and the exact modes bit for bit, because those traversals run one query per lane
in the same order; warp-coherent closest points and silhouettes with the same validity
and distance, and the same primitive except at FP32 distance ties, because a warp's
visit order depends on which queries share it.  The exact mode is also checked
against the CPU oracle.
"""
import math

import numpy as np
import pytest
import torch

import oracle
from gquery_b200 import _lib as L
from gquery_b200 import workloads as W
from gquery_b200.batch import SKIP, SceneBatch
from gquery_b200.scene import Scene
from parity import REL_TOL, assert_bitwise, tie_report, to_np

pytestmark = pytest.mark.gpu

CP2 = ["valid", "p", "n", "t", "d", "prim_id"]
CP3 = ["valid", "p", "n", "uv", "d", "prim_id"]
RAY2 = ["valid", "p", "n", "t", "d", "prim_id", "on_boundary"]
RAY3 = ["valid", "p", "n", "uv", "d", "prim_id", "on_boundary"]
SIL = ["valid", "p", "d", "prim_id"]


def _uneven_2d(n_scenes=12, seed=0):
    rng = np.random.default_rng(seed)
    scenes, geo = [], []
    for sid in range(n_scenes):
        m = int(round(math.exp(rng.uniform(math.log(16), math.log(20000)))))
        v, e = W.star_polyline(m, seed=100 + sid)
        scenes.append(Scene(v, e, 2, device=0, build_snch=True))
        geo.append((v, e))
    return scenes, geo


def _uneven_3d(seed=0):
    scenes, geo = [], []
    for lvl, amp, sd in [(1, 0.2, 1), (3, 0.3, 2), (5, 0.15, 3), (2, 0.0, 4), (4, 0.25, 5)]:
        v, f = W.icosphere(lvl, amplitude=amp, seed=sd)
        scenes.append(Scene(v, f, 3, device=0, build_snch=True))
        geo.append((v, f))
    return scenes, geo


def _mixed_queries(n, dim, n_scenes, seed):
    rng = np.random.default_rng(seed)
    ids = rng.integers(0, n_scenes, size=n).astype(np.int32)
    pts = rng.uniform(-2.0, 2.0, size=(n, dim)).astype(np.float32)
    d = rng.standard_normal((n, dim))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return ids, pts, d.astype(np.float32)


def _alone(scenes, ids, fn):
    """Runs each scene's queries alone and scatters the records back in query order."""
    out = None
    for sid, sc in enumerate(scenes):
        sel = np.nonzero(ids == sid)[0]
        if sel.size == 0:
            continue
        rec = to_np(fn(sc, sel))
        if out is None:
            out = {k: np.zeros(v.shape[:-1] + (ids.size,), v.dtype) for k, v in rec.items()}
        for k, v in rec.items():
            out[k][..., sel] = v
    return out


def _dev(x):
    return torch.as_tensor(x).cuda()


@pytest.fixture(scope="module")
def two_d():
    return _uneven_2d()


@pytest.fixture(scope="module")
def three_d():
    return _uneven_3d()


@pytest.mark.parametrize("dim", [2, 3])
def test_batch_matches_single_scene_calls(dim, two_d, three_d):
    scenes, _ = two_d if dim == 2 else three_d
    n = 40_000
    ids, pts, dirs = _mixed_queries(n, dim, len(scenes), seed=dim)
    cpf, rayf = (CP2, RAY2) if dim == 2 else (CP3, RAY3)
    b = SceneBatch(scenes, n)
    res = b.run(cp=(_dev(pts), _dev(ids)), ray=(_dev(pts), _dev(dirs), _dev(ids)), sil=(_dev(pts), _dev(ids)))
    torch.cuda.synchronize()
    assert b.device_error() == 0
    ray_alone = _alone(scenes, ids, lambda s, sel: s.intersect(_dev(pts[sel]), _dev(dirs[sel]), variant="wide8"))
    assert_bitwise(to_np(res.ray), ray_alone, rayf, "ray ")
    sil_alone = _alone(scenes, ids, lambda s, sel: s.closest_silhouette(_dev(pts[sel]), variant="coherent"))
    rep = tie_report(to_np(res.sil), sil_alone)
    assert rep["valid_mismatch"] == 0 and rep["prim_mismatch_not_tie"] == 0, rep
    assert rep["max_rel_d"] <= REL_TOL, rep
    cp_alone = _alone(scenes, ids, lambda s, sel: s.closest_point(_dev(pts[sel]), variant="coherent"))
    rep = tie_report(to_np(res.cp), cp_alone)
    assert rep["valid_mismatch"] == 0 and rep["prim_mismatch_not_tie"] == 0, rep
    assert rep["max_rel_d"] <= REL_TOL, rep
    exact = _alone(scenes, ids, lambda s, sel: s.closest_point(_dev(pts[sel]), variant="exact"))
    rep = tie_report(to_np(res.cp), exact)
    assert rep["valid_mismatch"] == 0 and rep["prim_mismatch_not_tie"] == 0, rep


@pytest.mark.parametrize("dim", [2, 3])
def test_batch_exact_mode_bitwise(dim, two_d, three_d):
    scenes, _ = two_d if dim == 2 else three_d
    n = 30_000
    ids, pts, dirs = _mixed_queries(n, dim, len(scenes), seed=10 + dim)
    cpf, rayf = (CP2, RAY2) if dim == 2 else (CP3, RAY3)
    b = SceneBatch(scenes, n, cp_variant="exact", ray_variant="exact", sil_variant="exact")
    res = b.run(cp=(_dev(pts), _dev(ids)), ray=(_dev(pts), _dev(dirs), _dev(ids), 1.5), sil=(_dev(pts), _dev(ids), 0.7))
    torch.cuda.synchronize()
    cp_alone = _alone(scenes, ids, lambda s, sel: s.closest_point(_dev(pts[sel]), variant="exact"))
    assert_bitwise(to_np(res.cp), cp_alone, cpf, "cp ")
    ray_alone = _alone(scenes, ids,
                       lambda s, sel: s.intersect(_dev(pts[sel]), _dev(dirs[sel]), 1.5, variant="exact"))
    assert_bitwise(to_np(res.ray), ray_alone, rayf, "ray ")
    sil_alone = _alone(scenes, ids, lambda s, sel: s.closest_silhouette(_dev(pts[sel]), 0.7, variant="exact"))
    assert_bitwise(to_np(res.sil), sil_alone, SIL, "sil ")


def test_batch_exact_mode_against_oracle(two_d):
    scenes, _ = two_d
    n = 4000
    ids, pts, _ = _mixed_queries(n, 2, len(scenes), seed=21)
    b = SceneBatch(scenes, n, cp_variant="exact")
    res = to_np(b.run(cp=(_dev(pts), _dev(ids))).cp)
    for sid, sc in enumerate(scenes):
        sel = np.nonzero(ids == sid)[0]
        if sel.size == 0:
            continue
        ref = oracle.closest_point(2, sc.ref_array(L.ARRAY_BVH_NODES), sc.ref_array(L.ARRAY_PRIMITIVES),
                                   pts[sel])
        got = {k: v[..., sel] for k, v in res.items()}
        assert_bitwise(got, ref, CP2, f"scene {sid} ")


def test_batch_padding_slots_untouched(three_d):
    scenes, _ = three_d
    n = 5000
    ids, pts, dirs = _mixed_queries(n, 3, len(scenes), seed=5)
    ids[::3] = SKIP
    b = SceneBatch(scenes, n)
    out = b.alloc(n, n, n)
    for rec in (out.cp, out.ray, out.sil):
        rec.d.fill_(-7.0)
        rec.prim_id.fill_(-7)
    res = b.run(cp=(_dev(pts), _dev(ids)), ray=(_dev(pts), _dev(dirs), _dev(ids)), sil=(_dev(pts), _dev(ids)),
                out=out)
    torch.cuda.synchronize()
    assert b.device_error() == 0
    pad = ids == SKIP
    for rec in (res.cp, res.ray, res.sil):
        d = rec.d.cpu().numpy()
        pid = rec.prim_id.cpu().numpy()
        assert np.all(d[pad] == -7.0) and np.all(pid[pad] == -7)
        assert not np.any(pid[~pad] == -7)


def test_batch_bad_scene_index_flags_error(three_d):
    scenes, _ = three_d
    n = 1000
    ids, pts, dirs = _mixed_queries(n, 3, len(scenes), seed=6)
    ids[17] = len(scenes) + 3
    ids[18] = -5
    b = SceneBatch(scenes, n)
    res = b.run(cp=(_dev(pts), _dev(ids)), ray=(_dev(pts), _dev(dirs), _dev(ids)), sil=(_dev(pts), _dev(ids)))
    torch.cuda.synchronize()
    flags = b.device_error()
    assert flags & L.BATCH_ERR_SCENE
    for rec in (res.cp, res.ray, res.sil):
        assert not rec.valid[17].item() and not rec.valid[18].item()
    assert b.device_error() == 0  # read clears


def test_batch_rejects_oversize_and_missing_snch():
    v, f = W.icosphere(2, seed=0)
    plain = Scene(v, f, 3, device=0, build_snch=False)
    b = SceneBatch([plain], 100)
    pts = torch.zeros(3, 200, device="cuda")
    ids = torch.zeros(200, dtype=torch.int32, device="cuda")
    with pytest.raises(L.GQError, match="max_queries"):
        b.run(cp=(pts, ids))
    with pytest.raises(L.GQError, match="SNCH"):
        b.run(sil=(pts[:, :50], ids[:50]))
    v2, e2 = W.star_polyline(64)
    with pytest.raises(L.GQError, match="dimension"):
        SceneBatch([plain, Scene(v2, e2, 2, device=0)], 10)


def test_batch_graph_replay_matches_eager(two_d):
    scenes, _ = two_d
    n_cp, n_ray, n_sil = 8192, 4096, 2048
    b = SceneBatch(scenes, 8192)
    g = b.capture(n_cp, n_ray, n_sil)
    for seed in (31, 32):
        ids, pts, dirs = _mixed_queries(n_cp, 2, len(scenes), seed=seed)
        g.cp_points.copy_(_dev(pts).t())
        g.cp_scene.copy_(_dev(ids))
        g.ray_origin.copy_(_dev(pts[:n_ray]).t())
        g.ray_dir.copy_(_dev(dirs[:n_ray]).t())
        g.ray_scene.copy_(_dev(ids[:n_ray]))
        g.sil_points.copy_(_dev(pts[:n_sil]).t())
        g.sil_scene.copy_(_dev(ids[:n_sil]))
        out = g.replay()
        torch.cuda.synchronize()
        eager = b.run(cp=(_dev(pts), _dev(ids)), ray=(_dev(pts[:n_ray]), _dev(dirs[:n_ray]), _dev(ids[:n_ray])),
                      sil=(_dev(pts[:n_sil]), _dev(ids[:n_sil])))
        torch.cuda.synchronize()
        assert_bitwise(to_np(out.cp), to_np(eager.cp), CP2, "cp ")
        assert_bitwise(to_np(out.ray), to_np(eager.ray), RAY2, "ray ")
        assert_bitwise(to_np(out.sil), to_np(eager.sil), SIL, "sil ")


def test_batch_single_kind_and_tiny(three_d):
    scenes, _ = three_d
    b = SceneBatch(scenes, 64)
    for n in (1, 31, 33):
        ids, pts, dirs = _mixed_queries(n, 3, len(scenes), seed=40 + n)
        res = b.run(ray=(_dev(pts), _dev(dirs), _dev(ids)))
        alone = _alone(scenes, ids, lambda s, sel: s.intersect(_dev(pts[sel]), _dev(dirs[sel]), variant="wide8"))
        assert_bitwise(to_np(res.ray), alone, RAY3, f"n={n} ")
    assert b.run().cp is None


@pytest.mark.parametrize("dim", [2, 3])
def test_batch_silhouettes_one_query_per_warp(dim, two_d, three_d):
    scenes, _ = two_d if dim == 2 else three_d
    n = 6000
    ids, pts, _ = _mixed_queries(n, dim, len(scenes), seed=50 + dim)
    ids[::11] = SKIP
    b = SceneBatch(scenes, n, sil_variant="warp")
    out = b.alloc(0, 0, n)
    out.sil.prim_id.fill_(-7)
    res = b.run(sil=(_dev(pts), _dev(ids), 0.9), out=out)
    torch.cuda.synchronize()
    assert b.device_error() == 0
    got = to_np(res.sil)
    live = ids != SKIP
    assert np.all(got["prim_id"][~live] == -7)
    ref = _alone(scenes, np.where(live, ids, -1),
                 lambda s, sel: s.closest_silhouette(_dev(pts[sel]), 0.9, variant="exact"))
    rep = tie_report({k: v[..., live] for k, v in got.items()}, {k: v[..., live] for k, v in ref.items()})
    assert rep["valid_mismatch"] == 0 and rep["prim_mismatch_not_tie"] == 0 and rep["max_rel_d"] <= REL_TOL, rep


@pytest.mark.parametrize("dim", [2, 3])
def test_batch_split_closest_points(dim, two_d, three_d):
    """cp_variant "split": one lane per query, long traversals restarted one per warp.
    An undisplaced sphere (circle) queried near its centre makes every primitive almost
    equally far, so those traversals pass the visit budget and take the warp path."""
    scenes, _ = two_d if dim == 2 else three_d
    if dim == 3:
        v, f = W.icosphere(5)
    else:
        t = np.linspace(0.0, 2.0 * np.pi, 20000, endpoint=False)
        v = np.stack([np.cos(t), np.sin(t)], 1).astype(np.float32)
        f = np.stack([np.arange(20000), (np.arange(20000) + 1) % 20000], 1).astype(np.int32)
    scenes = scenes + [Scene(v, f, dim, device=0, build_snch=False)]
    n = 6000
    ids, pts, _ = _mixed_queries(n, dim, len(scenes), seed=60 + dim)
    rng = np.random.default_rng(61)
    centre = slice(0, 1500)  # near the centre of the sphere / circle
    ids[centre] = len(scenes) - 1
    pts[centre] = rng.uniform(-0.02, 0.02, size=(1500, dim)).astype(np.float32)
    ids[::13] = SKIP
    b = SceneBatch(scenes, n, cp_variant="split")
    out = b.alloc(n, 0, 0)
    out.cp.prim_id.fill_(-7)
    res = b.run(cp=(_dev(pts), _dev(ids)), out=out)
    torch.cuda.synchronize()
    assert b.device_error() == 0
    got = to_np(res.cp)
    live = ids != SKIP
    assert np.all(got["prim_id"][~live] == -7)
    ref = _alone(scenes, np.where(live, ids, -1), lambda s, sel: s.closest_point(_dev(pts[sel]), variant="exact"))
    rep = tie_report({k: v[..., live] for k, v in got.items()}, {k: v[..., live] for k, v in ref.items()})
    assert rep["valid_mismatch"] == 0 and rep["prim_mismatch_not_tie"] == 0 and rep["max_rel_d"] <= REL_TOL, rep
    # a second run gives the same answers (the hand-over list and its counters restart)
    again = to_np(b.run(cp=(_dev(pts), _dev(ids))).cp)
    for k in ("valid", "d", "prim_id"):
        assert np.array_equal(again[k][..., live], got[k][..., live]), k


def test_batch_split_silhouettes():
    """sil_variant "split": one lane per query, traversals past 2048 steps taken over by
    one warp from the r_max they reached.  On this level-6 mesh about one uniform query
    in a thousand runs that long."""
    v, f = W.icosphere(6, amplitude=0.15, seed=5)
    scenes = [Scene(v, f, 3, device=0, build_snch=True)]
    n = 8000
    pts = W.uniform_points(n, 3, seed=3)
    ids = np.zeros(n, np.int32)
    ids[::17] = SKIP
    b = SceneBatch(scenes, n, sil_variant="split")
    out = b.alloc(0, 0, n)
    out.sil.prim_id.fill_(-7)
    res = b.run(sil=(_dev(pts), _dev(ids)), out=out)
    torch.cuda.synchronize()
    assert b.device_error() == 0
    got = to_np(res.sil)
    live = ids != SKIP
    assert np.all(got["prim_id"][~live] == -7)
    ref = to_np(scenes[0].closest_silhouette(_dev(pts[live]), variant="exact"))
    rep = tie_report({k: v[..., live] for k, v in got.items()}, ref)
    assert rep["valid_mismatch"] == 0 and rep["prim_mismatch_not_tie"] == 0 and rep["max_rel_d"] <= REL_TOL, rep
    again = to_np(b.run(sil=(_dev(pts), _dev(ids))).sil)
    for k in ("valid", "d", "prim_id"):
        assert np.array_equal(again[k][..., live], got[k][..., live]), k
