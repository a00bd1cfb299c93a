"""The device-side stack bound, made to run out on purpose.

A scene's traversal stacks are capped below what its tree needs
(gq_scene_set_stack_limit).  Every kernel must then stop the walks that would push past
the cap, return normally, write those queries as zeroed misses, raise GQ_DEVERR_STACK in
the error word, and answer every other query exactly as without the cap.  Nothing here
traps, faults or waits: the bound is a plain comparison before each push."""
import numpy as np
import pytest
import torch

from gquery_b200 import _lib as L
from gquery_b200 import workloads as W
from gquery_b200.batch import SceneBatch
from gquery_b200.scene import Scene
from parity import assert_bitwise, to_np

pytestmark = pytest.mark.gpu

FIELDS = {"cp": ["valid", "p", "n", "uv", "d", "prim_id"], "ray": ["valid", "p", "n", "uv", "d", "prim_id", "on_boundary"],
          "sil": ["valid", "p", "d", "prim_id"]}
CAP = 3


@pytest.fixture(scope="module")
def mesh():
    v, f = W.icosphere(4, amplitude=0.3, seed=3)
    return Scene(v, f, 3, device=0, build_snch=True)


@pytest.fixture(scope="module")
def queries():
    q = W.uniform_points(20_000, 3, seed=61)
    o, d = W.rays(20_000, 3, seed=62)
    return torch.as_tensor(q).cuda(), torch.as_tensor(o).cuda(), torch.as_tensor(d).cuda()


def _call(s, kind, variant, qs):
    q, o, d = qs
    if variant == "wide8_group":  # one ray per group of 8 lanes
        s.set_tuning("ray", "wide8", packet=1)
        try:
            return to_np(s.intersect(o, d, variant="wide8"))
        finally:
            s.set_tuning("ray", "wide8", packet=0)
    if kind == "cp":
        return to_np(s.closest_point(q, variant=variant))
    if kind == "ray":
        return to_np(s.intersect(o, d, variant=variant))
    return to_np(s.closest_silhouette(q, variant=variant))


def _check_stopped(capped, free, fields, what):
    """Queries the capped run answered equal the uncapped answers bit for bit; the rest
    are zeroed misses.  Returns the number of stopped queries."""
    v = capped["valid"].astype(bool)
    kept = {k: np.asarray(x)[..., v] for k, x in capped.items()}
    assert_bitwise(kept, {k: np.asarray(x)[..., v] for k, x in free.items()}, fields, what)
    for k in fields:
        x = np.asarray(capped[k])[..., ~v]
        assert not np.any(x.astype(np.float64) != 0), f"{what}{k}: a stopped query is not a zeroed miss"
    return int(np.count_nonzero(free["valid"].astype(bool) & ~v))


@pytest.mark.parametrize("kind,variant", [("cp", "exact"), ("cp", "coherent"), ("cp", "wide8"), ("ray", "exact"),
                                          ("ray", "wide8"), ("ray", "wide8_group"), ("sil", "exact"),
                                          ("sil", "coherent")])
def test_single_scene_overflow_is_flagged_and_zeroed(mesh, queries, kind, variant):
    mesh.set_stack_limit(0)
    free = _call(mesh, kind, variant, queries)
    assert mesh.device_error() == 0
    mesh.set_stack_limit(CAP)
    try:
        capped = _call(mesh, kind, variant, queries)
        err = mesh.device_error()  # the call returned; read and clear the word
    finally:
        mesh.set_stack_limit(0)
    assert err & L.DEVERR_STACK, f"{kind}/{variant}: stack bit not raised (error word {err})"
    stopped = _check_stopped(capped, free, FIELDS[kind], f"{kind}/{variant} ")
    assert stopped > 0
    # the word was cleared and the uncapped scene answers as before
    again = _call(mesh, kind, variant, queries)
    assert mesh.device_error() == 0
    assert_bitwise(again, free, FIELDS[kind], f"{kind}/{variant} after reset ")


def test_batch_overflow_is_flagged_and_zeroed(mesh, queries):
    q, o, d = queries
    ids = torch.zeros(q.shape[0], dtype=torch.int32, device=q.device)
    free_batch = SceneBatch([mesh], q.shape[0], cp_variant="exact", ray_variant="exact", sil_variant="exact")
    free = free_batch.run(cp=(q, ids), ray=(o, d, ids), sil=(q, ids))
    torch.cuda.synchronize()
    assert free_batch.device_error() == 0
    mesh.set_stack_limit(CAP)
    try:
        capped_batch = SceneBatch([mesh], q.shape[0], cp_variant="exact", ray_variant="exact", sil_variant="exact")
    finally:
        mesh.set_stack_limit(0)  # the batch keeps the cap it was created with
    res = capped_batch.run(cp=(q, ids), ray=(o, d, ids), sil=(q, ids))
    err = capped_batch.device_error()
    assert err & L.DEVERR_STACK, err
    for kind, a, b in (("cp", res.cp, free.cp), ("ray", res.ray, free.ray), ("sil", res.sil, free.sil)):
        assert _check_stopped(to_np(a), to_np(b), FIELDS[kind], f"batch {kind} ") > 0
    # a scene's own calls are unaffected by the batch's copy of the cap
    assert_bitwise(to_np(mesh.closest_point(q, variant="exact")), to_np(free.cp), FIELDS["cp"], "scene after batch ")
    assert capped_batch.device_error() == 0 and mesh.device_error() == 0


def test_stack_limit_rejects_negative(mesh):
    with pytest.raises(Exception):
        mesh.set_stack_limit(-1)
