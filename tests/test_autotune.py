"""Autotuner on the GPU: every candidate launch configuration (node width, stack depth,
block shape, refill budget) gives the exact traversal's answers up to FP32 ties, and
the tuned choice lands in the scene's table."""
import numpy as np
import pytest
import torch

from gquery_b200 import workloads as W
from gquery_b200.autotune import TuneCache, candidates, tune
from gquery_b200.scene import Scene
from parity import REL_TOL, tie_report, to_np

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mesh():
    v, f = W.icosphere(5, amplitude=0.25, seed=8)
    return Scene(v, f, 3, device=0, build_snch=True)


@pytest.mark.parametrize("kind", ["cp", "ray", "sil"])
def test_every_candidate_agrees_and_best_is_applied(mesh, kind, tmp_path):
    n = 20000
    q = torch.as_tensor(W.uniform_points(n, 3, seed=81)).cuda()
    o, d = (torch.as_tensor(a).cuda() for a in W.rays(n, 3, seed=82))
    inputs = {"cp": (q,), "ray": (o, d), "sil": (q,)}[kind]
    cache = TuneCache(str(tmp_path / "t.json"))
    res = tune(mesh, kind, inputs, cache=cache)
    info = mesh.info
    assert len(res.table) == len(candidates(kind, 3, True, info["exact_stack"], info["wide_stack"]))
    assert all(t["agrees"] for t in res.table), [t for t in res.table if not t["agrees"]]
    got = mesh.get_tuning(kind)
    for k, v in res.best.items():
        assert got[k] == v, (k, got, res.best)
    # answers under the tuned table equal the exact ones up to ties
    run = {"cp": lambda v: mesh.closest_point(q, variant=v), "ray": lambda v: mesh.intersect(o, d, variant=v),
           "sil": lambda v: mesh.closest_silhouette(q, variant=v)}[kind]
    rep = tie_report(to_np(run("exact")), to_np(run("auto")))
    assert rep["valid_mismatch"] == 0 and rep["prim_mismatch_not_tie"] == 0 and rep["max_rel_d"] <= REL_TOL, rep
    assert tune(mesh, kind, inputs, cache=cache).from_cache
    assert mesh.device_error() == 0


def test_short_stack_and_block_sizes_bitwise_equal_for_coherent(mesh):
    q = torch.as_tensor(W.uniform_points(30000, 3, seed=83)).cuda()
    saved = mesh.get_tuning("cp")
    try:
        outs = []
        for block, stack in ((128, 0), (64, 32), (256, 32), (256, 0)):
            mesh.set_tuning("cp", "coherent", packet=1, block=block, stack=stack)
            outs.append(to_np(mesh.closest_point(q, variant="auto")))
        for o in outs[1:]:
            for k in ("valid", "d", "prim_id"):
                assert np.array_equal(np.asarray(o[k]), np.asarray(outs[0][k])), k
    finally:
        mesh.set_tuning("cp", **saved)
    with pytest.raises(Exception, match="block"):
        mesh.set_tuning("cp", "coherent", block=96)
