"""gq_closest_point_noalloc: closest point without device allocation, for callers that
cannot allocate while they query (a plugin whose host application owns all device
memory, a real-time loop that must not enter an allocator).  Its scratch is a fixed
array in the library, shared by all calls on a device.

Checked through the C ABI against gq_closest_point on the same inputs, for two calls in
a row (the second call must not see leftovers of the first), plus the size limit.
This file sorts last so a failure here stops a run only after every other test ran."""
import ctypes as C

import numpy as np
import pytest
import torch

from gquery_b200 import _lib as L
from gquery_b200 import workloads as W
from gquery_b200.scene import Scene, points_layout

pytestmark = pytest.mark.gpu

REL_TOL = 2e-6


def _call_noalloc(scene, q, variant, sort):
    t, n, cs, es = points_layout(q, scene.dim)
    rec = scene.alloc_cp(n)
    out = scene.cp_out_struct(rec)
    st = L.lib().gq_closest_point_noalloc(scene.handle, L.Vecs(t.data_ptr(), cs, es), n, C.byref(out), variant,
                                          int(sort), torch.cuda.current_stream().cuda_stream)
    L.check(st)
    return rec


def _np(rec):
    return {k: v.cpu().numpy() for k, v in vars(rec).items()}


@pytest.fixture(scope="module")
def scene():
    v, f = W.icosphere(6, amplitude=0.15, seed=0)
    return Scene(v, f, 3, device=0, build_snch=False)


@pytest.fixture(scope="module")
def polyline():
    v, e = W.star_polyline(4096, seed=0)
    return Scene(v, e, 2, device=0, build_snch=False)


def _compare(got, ref, fields):
    assert np.array_equal(got["valid"], ref["valid"])
    assert np.array_equal(got["prim_id"], ref["prim_id"])
    for f in fields:
        np.testing.assert_allclose(got[f], ref[f], rtol=REL_TOL, atol=0)


@pytest.mark.parametrize("variant", [L.VARIANT_COHERENT, L.VARIANT_WIDE8, L.VARIANT_EXACT])
def test_noalloc_matches_allocating_entry_point_twice(scene, variant):
    cap = L.lib().gq_noalloc_max_queries()
    assert cap >= 32768
    name = {L.VARIANT_COHERENT: "coherent", L.VARIANT_WIDE8: "wide8", L.VARIANT_EXACT: "exact"}[variant]
    for call, n in enumerate((cap, 20000)):
        q = torch.as_tensor(W.uniform_points(n, 3, seed=100 + call)).cuda()
        got = _np(_call_noalloc(scene, q, variant, sort=True))
        ref = _np(scene.closest_point(q, variant=name, sort=True))
        _compare(got, ref, ("p", "n", "uv", "d"))
    assert scene.device_error() == 0


@pytest.mark.parametrize("sort", [False, True])
@pytest.mark.parametrize("variant", [L.VARIANT_COHERENT, L.VARIANT_EXACT])
def test_noalloc_polyline_sorted_and_unsorted(polyline, variant, sort):
    cap = L.lib().gq_noalloc_max_queries()
    name = {L.VARIANT_COHERENT: "coherent", L.VARIANT_EXACT: "exact"}[variant]
    for call, n in enumerate((cap, 777)):
        q = torch.as_tensor(W.uniform_points(n, 2, seed=200 + call)).cuda()
        got = _np(_call_noalloc(polyline, q, variant, sort=sort))
        ref = _np(polyline.closest_point(q, variant=name, sort=sort))
        _compare(got, ref, ("p", "n", "t", "d"))
    assert polyline.device_error() == 0


def test_noalloc_rejects_oversized_batches(scene):
    cap = L.lib().gq_noalloc_max_queries()
    q = torch.zeros((cap + 1, 3), dtype=torch.float32, device="cuda")
    t, n, cs, es = points_layout(q, 3)
    rec = scene.alloc_cp(n)
    out = scene.cp_out_struct(rec)
    st = L.lib().gq_closest_point_noalloc(scene.handle, L.Vecs(t.data_ptr(), cs, es), n, C.byref(out),
                                          L.VARIANT_COHERENT, 1, torch.cuda.current_stream().cuda_stream)
    assert st == L.GQ_ERR_INVALID
    assert "at most" in L.last_error()
