"""Host-side pieces of the serving layer: load generation, request records, summaries."""
import ctypes as C

import numpy as np

from gquery_b200 import _lib as L
from gquery_b200.serving import HostRequest, poisson_arrivals, request_mix, result_fields, summarize


def test_poisson_arrivals_rate_and_order():
    rng = np.random.default_rng(0)
    t = poisson_arrivals(5000.0, 20000, rng)
    assert np.all(np.diff(t) >= 0)
    assert abs(20000 / t[-1] - 5000.0) / 5000.0 < 0.03
    assert np.all(poisson_arrivals(float("inf"), 5, rng) == 0)


def test_request_mix_bounds_and_shares():
    rng = np.random.default_rng(1)
    sc, kinds, counts = request_mix(50000, 64, rng, max_queries=262144)
    assert sc.min() >= 0 and sc.max() == 63
    assert counts.min() >= 1 and counts.max() <= 262144
    share = np.bincount(kinds, minlength=3) / kinds.size
    assert np.allclose(share, [0.5, 0.3, 0.2], atol=0.01)
    # log-uniform: about half the requests below sqrt(262144) = 512
    assert 0.45 < np.mean(counts < 512) < 0.55


def test_result_fields_follow_reference_records():
    assert list(result_fields("cp", 3)) == ["valid", "p", "n", "uv", "d", "prim_id"]
    assert list(result_fields("cp", 2)) == ["valid", "p", "n", "t", "d", "prim_id"]
    assert list(result_fields("ray", 3))[-1] == "on_boundary"
    assert list(result_fields("sil", 3)) == ["valid", "p", "d", "prim_id"]


def test_host_request_struct_points_at_its_arrays():
    a = np.arange(30, dtype=np.float32).reshape(10, 3)
    r = HostRequest.make(2, "ray", a, a[::-1], None)
    s = r.struct()
    assert s.n == 10 and s.scene == 2 and s.kind == L.KIND_INTERSECT
    assert s.a == r.a.ctypes.data and s.b == r.b.ctypes.data and not s.r_max
    assert s.ray_out.p == r.out["p"].ctypes.data and r.out["p"].shape == (3, 10)
    assert s.ray_out.t == r.out["uv"].ctypes.data and r.out["uv"].shape == (2, 10)
    assert not s.cp_out.p and not s.sil_out.p
    assert C.sizeof(L.Request) == 8 + 8 + 3 * 8 + 6 * 8 + 7 * 8 + 4 * 8 + 8


def test_summarize_percentiles_and_throughput():
    n = 1000
    t_sub = np.linspace(0.0, 1.0, n)
    lat = np.full(n, 0.002)
    lat[-10:] = 0.010
    res = {"t_submit": t_sub, "t_done": t_sub + lat, "n": np.full(n, 1000), "step": np.arange(n) // 4}
    s = summarize(res)
    assert abs(s["p50_ms"] - 2.0) < 1e-9 and s["max_ms"] > 9.99
    assert abs(s["mqueries_per_s"] - 1e6 / 1.010 / 1e6) < 1e-9
    assert s["steps"] == 250


def test_place_scenes_respects_budgets_and_balances():
    from gquery_b200.serving import place_scenes
    sizes = [50, 40, 30, 20, 10, 10]
    place = place_scenes(sizes, [80, 100])
    used = [sum(s for s, p in zip(sizes, place) if p == d) for d in range(2)]
    assert used[0] <= 80 and used[1] <= 100 and sum(used) == sum(sizes)
    assert place[0] != place[1]  # the two largest go to different devices
    assert place_scenes([5, 5], [10]) == [0, 0]
    import pytest
    with pytest.raises(ValueError, match="fits on no device"):
        place_scenes([60, 60], [50, 100])
    with pytest.raises(ValueError):
        place_scenes([1], [])
