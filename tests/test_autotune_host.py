"""Autotuner logic on the host: candidates, selection, verification and the cache, with
a stand-in scene whose timings and answers are scripted."""
import math
import types

import numpy as np
import pytest

from gquery_b200.autotune import BATCH_CHOICES, TuneCache, candidates, config_key, full_config, tune, tune_batch


def test_candidates_cover_width_stack_and_block():
    c = candidates("cp", 3, True, 24, 40)
    keys = {config_key(x) for x in c}
    assert len(keys) == len(c)
    assert {x["variant"] for x in c} == {"exact", "coherent", "wide8"}
    assert {x["block"] for x in c} == {64, 128, 256}
    assert any(x["stack"] == 32 for x in c)
    assert not any(x["stack"] == 32 for x in candidates("cp", 3, True, 40, 60))
    assert all(x["variant"] != "wide8" for x in candidates("cp", 3, False, 24, 0))
    assert candidates("sil", 3, True, 24, 40, has_snch=False) == []
    assert {x["variant"] for x in candidates("sil", 2, True, 20, 20)} == {"coherent", "exact", "warp"}


class FakeScene:
    """Answers depend on the tuned variant; 'wide8' is made to disagree on purpose."""

    def __init__(self):
        self.dim = 3
        self.info = dict(dim=3, n_prims=1000, n_nodes=199, n_wide_nodes=40, exact_stack=20, wide_stack=30,
                         n_silhouettes=10)
        self.tuning = {k: full_config({}) for k in ("cp", "ray", "sil")}
        self.calls = 0

    def set_tuning(self, kind, **kw):
        self.tuning[kind] = full_config(kw)

    def get_tuning(self, kind):
        return dict(self.tuning[kind])

    def closest_point(self, q, variant="auto"):
        self.calls += 1
        v = self.tuning["cp"]["variant"] if variant == "auto" else variant
        d = np.linspace(0.1, 1.0, 8).astype(np.float32)
        if v == "wide8":
            d = d * 1.01
        return types.SimpleNamespace(valid=np.ones(8, bool), d=d, prim_id=np.arange(8))


def test_tune_picks_fastest_agreeing_and_caches(tmp_path):
    sc = FakeScene()
    speed = {"exact": 5.0, "coherent": 2.0, "wide8": 1.0}  # wide8 fastest but wrong

    def timer(fn):
        fn()
        c = sc.tuning["cp"]
        return speed[c["variant"]] + c["block"] / 1000.0 + (0.5 if c["stack"] == 0 else 0.0)

    q = np.zeros((8, 3), np.float32)
    cache = TuneCache(str(tmp_path / "tune.json"))
    res = tune(sc, "cp", (q,), timer=timer, cache=cache)
    assert res.best["variant"] == "coherent" and res.best["block"] == 64 and res.best["stack"] == 32
    assert any(not t["agrees"] and math.isinf(t["ms"]) for t in res.table)
    assert sc.tuning["cp"] == res.best
    sc2 = FakeScene()
    res2 = tune(sc2, "cp", (q,), timer=timer, cache=TuneCache(str(tmp_path / "tune.json")))
    assert res2.from_cache and sc2.tuning["cp"] == res.best and sc2.calls == 0


def test_tune_restores_table_when_nothing_agrees():
    sc = FakeScene()
    with pytest.raises(RuntimeError):
        tune(sc, "cp", (np.zeros((8, 3), np.float32),), cands=[full_config(dict(variant="wide8"))],
             timer=lambda fn: 1.0)
    assert sc.tuning["cp"] == full_config({})


def test_tune_batch_picks_fastest_choice():
    made = []

    def make(**ch):
        made.append(ch)
        return ch

    t = {("coherent", "wide8", "coherent"): 1.0}
    res = tune_batch(make, lambda b: None, timer=lambda fn: t.get(tuple(made[-1].values()), 2.0))
    assert res["best"] == dict(cp_variant="coherent", ray_variant="wide8", sil_variant="coherent")
    assert len(res["table"]) == len(BATCH_CHOICES) == 18
