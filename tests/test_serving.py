"""Serving runtime (gq_server_*): continuous batching with admission by memory budget.

The central property: a request's result does not depend on what it was batched with.
Rays must equal the single-scene call on the same queries bit for bit; warp-coherent
closest points and silhouettes must have the same validity and distances and the same
primitive except at FP32 distance ties (a warp's visit order depends on which queries
share it).  The plain per-request mode must equal the
single-scene call too.
"""
import threading

import numpy as np
import pytest
import torch

from gquery_b200 import _lib as L
from gquery_b200 import workloads as W
from gquery_b200.scene import Scene
from gquery_b200.serving import HostRequest, Server, poisson_arrivals, request_mix, summarize
from parity import REL_TOL, assert_bitwise, tie_report, to_np

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scenes():
    out = []
    for lvl, amp, sd in [(2, 0.2, 1), (4, 0.3, 2), (5, 0.15, 3), (3, 0.0, 4)]:
        v, f = W.icosphere(lvl, amplitude=amp, seed=sd)
        out.append(Scene(v, f, 3, device=0, build_snch=True))
    return out


def _requests(n_req, n_scenes, seed, max_q=3000):
    rng = np.random.default_rng(seed)
    sc, kinds, counts = request_mix(n_req, n_scenes, rng, max_queries=max_q)
    reqs = []
    for s, k, c in zip(sc, kinds, counts):
        pts = rng.uniform(-2.0, 2.0, size=(c, 3)).astype(np.float32)
        d = rng.standard_normal((c, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        kind = ("cp", "ray", "sil")[k]
        rmax = None
        if kind != "cp" and rng.random() < 0.3:
            rmax = rng.uniform(0.2, 3.0, size=c).astype(np.float32)
        reqs.append(HostRequest.make(int(s), kind, pts, d.astype(np.float32) if kind == "ray" else None, rmax))
    return reqs


def _soa(x):
    # [D, n] on the device: unambiguous even when n == D
    return torch.as_tensor(np.ascontiguousarray(x.T)).cuda()


def _alone(scene, req):
    a = _soa(req.a)
    r = np.inf if req.r_max is None else torch.as_tensor(req.r_max).cuda()
    if req.kind == "cp":
        return to_np(scene.closest_point(a, variant="coherent"))
    if req.kind == "ray":
        return to_np(scene.intersect(a, _soa(req.b), r, variant="wide8"))
    return to_np(scene.closest_silhouette(a, r, variant="coherent"))


def _check_same_as_alone(scenes, reqs):
    for i, req in enumerate(reqs):
        assert req.completion is not None and req.completion["status"] == 0, i
        ref = _alone(scenes[req.scene], req)
        got = dict(req.out)
        if req.kind in ("cp", "sil"):
            rep = tie_report(got, ref)
            assert rep["valid_mismatch"] == 0 and rep["prim_mismatch_not_tie"] == 0, (i, req.n, rep)
            assert rep["max_rel_d"] <= REL_TOL, (i, rep)
        else:
            assert_bitwise(got, ref, list(req.out.keys()), f"request {i} ({req.kind}, n={req.n}) ")


def test_results_same_alone_and_in_the_mix(scenes):
    reqs = _requests(160, len(scenes), seed=1)
    srv = Server(scenes, ring_queries=(1 << 16,) * 3, step_queries=1 << 14, max_inflight=2)
    # everything arrives within about 2 ms, so requests share steps
    res = srv.run_trace(reqs, poisson_arrivals(80_000.0, len(reqs), np.random.default_rng(2)))
    st = srv.stats()
    assert st["device_error"] == 0 and st["requests_done"] == len(reqs)
    _, per_step = np.unique(res["step"], return_counts=True)
    assert per_step.max() > 1, "no step served more than one request"
    _check_same_as_alone(scenes, reqs)


@pytest.mark.parametrize("cp_variant,sil_variant", [("split", "warp"), ("coherent", "coherent")])
def test_large_class_steps_hold_one_class(scenes, cp_variant, sil_variant):
    # requests of >= 1000 queries are large: their own rings, steps and slots; a few of
    # 40-70 K queries make the host copies run on the copy threads.  Small steps are not
    # sorted, so the warp-coherent forms see queries of several scenes in one tile.
    reqs = _requests(150, len(scenes), seed=12)
    rng = np.random.default_rng(14)
    for i, kind in enumerate(("cp", "ray", "sil", "cp", "sil", "ray")):
        c = int(rng.integers(40_000, 70_000))
        pts = rng.uniform(-2.0, 2.0, size=(c, 3)).astype(np.float32)
        d = rng.standard_normal((c, 3))
        d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
        reqs.insert(20 * i + 5, HostRequest.make(i % len(scenes), kind, pts, d if kind == "ray" else None))
    srv = Server(scenes, ring_queries=(1 << 18,) * 3, step_queries=1 << 17, max_inflight=2, large_queries=1000,
                 cp_variant=cp_variant, sil_variant=sil_variant)
    res = srv.run_trace(reqs, poisson_arrivals(60_000.0, len(reqs), np.random.default_rng(13)))
    st = srv.stats()
    assert st["device_error"] == 0 and st["requests_done"] == len(reqs)
    large = res["n"] >= 1000
    assert large.any() and (~large).any()
    assert st["large_queries"] == 1000
    steps, per_step = np.unique(res["step"], return_counts=True)
    for s in steps:
        m = res["step"] == s
        assert large[m].all() or not large[m].any(), f"step {s} mixes size classes"
    assert per_step.max() > 1, "no step served more than one request"
    _check_same_as_alone(scenes, reqs)
    srv.close()


def test_size_classes_only_where_half_rings_hold_a_largest_request(scenes):
    # halves of 2,048 slots cannot hold a 4,096-query request: one class, all of the ring
    one = Server(scenes, ring_queries=(4096,) * 3, step_queries=4096, large_queries=1000)
    two = Server(scenes, ring_queries=(8192,) * 3, step_queries=4096, large_queries=1000)
    plain = Server(scenes, ring_queries=(8192,) * 3, step_queries=4096, large_queries=1000, per_request=True)
    try:
        assert one.stats()["large_queries"] == 0
        assert two.stats()["large_queries"] == 1000
        assert plain.stats()["large_queries"] == 0
        big = HostRequest.make(0, "cp", np.zeros((4096, 3), np.float32))
        one.submit(big)  # fits the single ring
        assert len(one.wait_idle(60.0)) == 1 and big.completion["status"] == 0
    finally:
        for s in (one, two, plain):
            s.close()


def test_per_request_mode_same_as_alone(scenes):
    reqs = _requests(40, len(scenes), seed=3)
    srv = Server(scenes, ring_queries=(1 << 16,) * 3, step_queries=1 << 14, per_request=True)
    res = srv.run_trace(reqs, np.zeros(len(reqs)))
    assert np.unique(res["step"]).size == len(reqs)
    assert srv.stats()["device_error"] == 0
    _check_same_as_alone(scenes, reqs)


def test_admission_waits_for_ring_space(scenes):
    # rings hold 4096 queries per kind; 200 requests of up to 3000 queries must queue
    reqs = _requests(200, len(scenes), seed=4)
    srv = Server(scenes, ring_queries=(4096, 4096, 4096), step_queries=4096)
    res = srv.run_trace(reqs, np.zeros(len(reqs)))
    st = srv.stats()
    assert st["requests_done"] == len(reqs) and st["device_error"] == 0
    assert st["admitted_bytes_peak"] <= st["device_bytes"]
    assert np.all(res["t_admit"] >= res["t_submit"]) and np.all(res["t_done"] >= res["t_launch"])
    assert np.all(res["status"] == 0)
    _check_same_as_alone(scenes, reqs[::7])


def test_budget_and_request_limits(scenes):
    with pytest.raises(L.GQError, match="budget"):
        Server(scenes, budget_bytes=1 << 20, ring_queries=(1 << 16,) * 3)
    srv = Server(scenes, ring_queries=(1024,) * 3, step_queries=1024)
    with pytest.raises(L.GQError, match="request size"):
        srv.submit(HostRequest.make(0, "cp", np.zeros((2000, 3), np.float32)))
    v, f = W.icosphere(2, seed=0)
    plain = Scene(v, f, 3, device=0, build_snch=False)
    srv2 = Server([plain], ring_queries=(1024,) * 3, step_queries=1024)
    with pytest.raises(L.GQError, match="SNCH"):
        srv2.submit(HostRequest.make(0, "sil", np.zeros((10, 3), np.float32)))
    with pytest.raises(L.GQError, match="scene index"):
        srv2.submit(HostRequest.make(3, "cp", np.zeros((10, 3), np.float32)))


def test_submit_from_threads_and_poll(scenes):
    reqs = _requests(60, len(scenes), seed=5)
    srv = Server(scenes, ring_queries=(1 << 15,) * 3, step_queries=1 << 13, max_inflight=3)

    def worker(part):
        for r in part:
            srv.submit(r)

    ts = [threading.Thread(target=worker, args=(reqs[i::3],)) for i in range(3)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    done = srv.wait_idle(60.0)
    assert len(done) == len(reqs)
    assert all(r.completion["status"] == 0 for r in done)
    _check_same_as_alone(scenes, reqs[::5])


def test_summary_of_a_short_open_loop_run(scenes):
    reqs = _requests(100, len(scenes), seed=6)
    srv = Server(scenes, ring_queries=(1 << 16,) * 3, step_queries=1 << 14)
    res = srv.run_trace(reqs, poisson_arrivals(2000.0, len(reqs), np.random.default_rng(7)))
    s = summarize(res)
    assert s["requests"] == len(reqs) and s["p99_ms"] >= s["p50_ms"] > 0
    assert s["queries"] == sum(r.n for r in reqs)


def test_router_sends_requests_to_their_scene(scenes):
    from gquery_b200.serving import Router, place_scenes
    assert place_scenes([s.info["device_bytes"] for s in scenes], [1 << 40]) == [0] * len(scenes)
    router = Router(scenes, ring_queries=(1 << 15,) * 3, step_queries=1 << 13)
    reqs = _requests(30, len(scenes), seed=11)
    for r in reqs:
        d, _ = router.submit(r)
        assert d == 0
    done = router.wait_idle(60.0)
    assert len(done) == len(reqs) and all(r.completion["status"] == 0 for r in done)
    _check_same_as_alone(scenes, reqs)
    with pytest.raises(ValueError):
        router.submit(HostRequest.make(len(scenes) + 1, "cp", np.zeros((4, 3), np.float32)))
    router.close()
