"""CPU builder checks: tree invariants, determinism, reference layouts, silhouettes,
normal cones and the outward rounding of the quantised wide nodes."""
import math

import numpy as np
import pytest

from gquery_b200 import _lib as L
from gquery_b200 import gquery_ext as gx
from gquery_b200 import workloads as W
from gquery_b200.scene import Scene


def _host(v, f, dim, **kw):
    return Scene(v, f, dim, device=None, **kw)


def _nodes(s):
    stride = 2 * s.dim + 3
    return s.ref_array(L.ARRAY_BVH_NODES).reshape(-1, stride)


def check_tree(s):
    D = s.dim
    N = _nodes(s)
    P = s.ref_array(L.ARRAY_PRIMITIVES).reshape(-1, D * D + 1)
    lo, hi = N[:, :D], N[:, D:2 * D]
    off, sco, cnt = N[:, 2 * D].astype(np.int64), N[:, 2 * D + 1].astype(np.int64), N[:, 2 * D + 2].astype(np.int64)
    seen = np.zeros(P.shape[0], np.int64)
    stack = [(0, len(N))]
    while stack:
        i, end = stack.pop()
        if cnt[i] > 0:
            assert sco[i] == 0
            seen[off[i]:off[i] + cnt[i]] += 1
            pv = P[off[i]:off[i] + cnt[i], :D * D].reshape(-1, D, D)
            assert (pv.min(axis=1) >= lo[i] - 1e-6).all() and (pv.max(axis=1) <= hi[i] + 1e-6).all()
        else:
            assert off[i] == 0 and 1 < sco[i] < end - i
            l, r = i + 1, i + sco[i]
            for c in (l, r):
                assert (lo[c] >= lo[i]).all() and (hi[c] <= hi[i]).all()
            assert np.array_equal(np.minimum(lo[l], lo[r]), lo[i])
            assert np.array_equal(np.maximum(hi[l], hi[r]), hi[i])
            stack.append((l, r))
            stack.append((r, end))
    assert (seen == 1).all(), "every ordered primitive belongs to exactly one leaf"
    assert sorted(P[:, -1].astype(np.int64).tolist()) == list(range(P.shape[0]))


def test_tree_invariants_2d():
    v, e = W.star_polyline(4096, seed=0)
    check_tree(_host(v, e, 2))


def test_tree_invariants_3d():
    v, f = W.icosphere(5, amplitude=0.2, seed=1)
    check_tree(_host(v, f, 3))


def test_leaf_sizes_bounded():
    v, f = W.icosphere(5, amplitude=0.2, seed=1)
    N = _nodes(_host(v, f, 3))
    cnt = N[:, 8]
    assert cnt.max() <= 10
    assert (cnt[cnt > 0] >= 1).all()


def test_build_deterministic_and_thread_count_independent():
    v, f = W.icosphere(6, amplitude=0.15, seed=0)
    a = _host(v, f, 3, n_threads=1)
    b = _host(v, f, 3, n_threads=8)
    c = _host(v, f, 3, n_threads=3)
    # the reference layouts, and the device records built from them (wide nodes, SNCH
    # pairs with their node bounds and searched cone axes, silhouette records)
    for which in (L.ARRAY_BVH_NODES, L.ARRAY_PRIMITIVES, L.ARRAY_SNCH_NODES, L.ARRAY_SILHOUETTES,
                  L.ARRAY_WIDE_NODES, L.ARRAY_SNCH_PAIRS, L.ARRAY_SIL_RECORDS):
        ra, rb, rc = a.ref_array(which), b.ref_array(which), c.ref_array(which)
        assert np.array_equal(ra.view(np.uint32), rb.view(np.uint32)), which
        assert np.array_equal(ra.view(np.uint32), rc.view(np.uint32)), which


def test_large_build_above_reference_thread_pool_threshold():
    # gQuery's builder throws above 131,072 primitives (its thread pool is never
    # initialised); this build must succeed and satisfy the invariants.
    v, f = W.icosphere(6, amplitude=0.15, seed=0)  # 81,920 faces
    v2 = np.concatenate([v, v + 3.0]).astype(np.float32)
    f2 = np.concatenate([f, f + v.shape[0]]).astype(np.int32)
    v3 = np.concatenate([v2, v2 + np.float32([0, 6, 0])]).astype(np.float32)
    f3 = np.concatenate([f2, f2 + v2.shape[0]]).astype(np.int32)
    s = _host(v3, f3, 3)
    assert s.info["n_prims"] == 327680
    check_tree(s)


def test_reference_layout_strides():
    v, e = W.star_polyline(512, seed=2)
    b = gx.SNCH(v, e)
    assert b.node_data().size % 13 == 0 and b.silhouette_data().size % 10 == 0
    assert b.primitive_data().size == 512 * 5
    assert gx.BVH(v, e).node_data().size % 7 == 0
    vv, ff = W.icosphere(3)
    b3 = gx.SNCH3D(vv, ff)
    assert b3.node_data().size % 16 == 0 and b3.silhouette_data().size % 19 == 0
    assert gx.BVH3D(vv, ff).node_data().size % 9 == 0
    assert gx.BVH3D(vv, ff).primitive_data().size == ff.shape[0] * 10


def test_soa_and_aos_inputs_build_the_same_tree():
    v, f = W.icosphere(3)
    a = gx.BVH3D(v, f).node_data()
    b = gx.BVH3D(v.T.copy(), f.T.copy()).node_data()
    assert np.array_equal(a, b)


def test_silhouette_edges_closed_mesh():
    v, f = W.icosphere(3)
    raw = gx.build_flat_silhouette_edges(v, f).reshape(-1, 19)
    n_edges = f.shape[0] * 3 // 2
    assert raw.shape[0] == n_edges
    # edge ids follow first appearance: ids are 0..E-1 in order
    assert np.array_equal(raw[:, 18], np.arange(n_edges, dtype=np.float32))
    # every edge's end points are its indices 1 and 2, sorted
    assert (raw[:, 13] < raw[:, 14]).all()
    # both faces recorded on a closed mesh, and the opposite vertices differ
    assert not np.array_equal(raw[:, 0:3], raw[:, 9:12])
    s = gx.SNCH3D(v, f)
    assert np.array_equal(s.raw_silhouette_data(), gx.build_flat_silhouette_edges(v, f))


def test_silhouette_edge_boundary_keeps_zero_vertex():
    # an open fan: boundary edges keep the value-initialised (0,0,0) fourth vertex
    v = np.array([[0, 0, 1], [1, 0, 1], [0, 1, 1], [-1, 0, 1]], np.float32)
    f = np.array([[0, 1, 2], [0, 2, 3]], np.int32)
    raw = gx.build_flat_silhouette_edges(v, f).reshape(-1, 19)
    boundary = [e for e in raw if not (e[12] != 0 and e[15] != 0)]
    assert len(boundary) >= 4
    for e in raw:
        if e[17] == 0 and e[16] == 0 and not np.any(e[9:12]):
            assert np.all(e[9:12] == 0)


def test_snch_cones_reference_rules():
    """Cones follow snch.cpp:103-154 over the node ranges the reference's recursion
    passes (snch.cpp:151-152): the root gets [0, n), a right child its parent's end, a
    left child its parent's RELATIVE second-child offset as its end.  A range without
    silhouettes leaves the invalid cone (half angle -pi, zero axis and radius); valid
    cones have unit axes (or the half angle pi)."""
    v, e = W.star_polyline(2048, seed=4)
    s = gx.SNCH(v, e)
    N = s.node_data().reshape(-1, 13)
    half, rad, axis = N[:, 6], N[:, 7], N[:, 4:6]
    second, nprim, nsil = N[:, 9].astype(np.int64), N[:, 10].astype(np.int64), N[:, 12].astype(np.int64)
    n = N.shape[0]
    end = np.zeros(n, np.int64)
    stack = [(0, n)]
    while stack:
        i, e_ = stack.pop()
        end[i] = e_
        if nprim[i] == 0:
            stack += [(i + 1, second[i]), (i + second[i], e_)]
    expect_valid = np.array([nsil[i:max(i, end[i])].sum() > 0 for i in range(n)])
    valid = half >= 0
    assert np.array_equal(valid, expect_valid)
    assert valid[0] and not valid.all()
    assert np.all(half[~valid] == np.float32(-math.pi))
    assert np.all(axis[~valid] == 0) and np.all(rad[~valid] == 0)
    norm = np.linalg.norm(axis, axis=1)
    assert np.allclose(norm[valid & (half < np.float32(math.pi))], 1.0, atol=1e-5)
    assert (rad >= 0).all()
    # the root's cone covers all silhouette normals of a closed star
    assert half[0] == np.float32(math.pi) or half[0] > 1.5


def test_snch_leaf_silhouettes_are_unique_within_leaf():
    v, f = W.icosphere(4, amplitude=0.3, seed=3)
    s = gx.SNCH3D(v, f)
    N = s.node_data().reshape(-1, 16)
    S = s.silhouette_data().reshape(-1, 19)
    for i in np.nonzero(N[:, 13] > 0)[0][:500]:
        off, n = int(N[i, 14]), int(N[i, 15])
        ids = S[off:off + n, 18]
        assert len(set(ids.tolist())) == n
        assert 3 <= n <= 30


def _decode_wide(words, dim):
    stride = 24 if dim == 3 else 20
    w = words.view(np.uint32).reshape(-1, stride)
    f = words.reshape(-1, stride)
    origin = f[:, :dim]
    meta = w[:, 3] if dim == 3 else w[:, 2]
    refs = w[:, 4:12].view(np.int32)
    q = w[:, 12:].copy().view(np.uint8).reshape(-1, 2 * dim, 8).astype(np.float32)
    exps = np.stack([(meta >> (8 * k)) & 0xff for k in range(dim)], axis=1).astype(np.int32) - 127
    nc = (meta >> 24).astype(np.int32)
    scale = np.ldexp(np.float32(1.0), exps).astype(np.float32)
    lo = np.empty((w.shape[0], 8, dim), np.float32)
    hi = np.empty_like(lo)
    for k in range(dim):  # decode like the kernels: fma(2^23 + q, 2^e, biased origin) in fp32
        s = scale[:, k:k + 1].astype(np.float64)
        o = origin[:, k:k + 1].astype(np.float64)
        lo[:, :, k] = ((q[:, k, :].astype(np.float64) + 8388608.0) * s + o).astype(np.float32)
        hi[:, :, k] = ((q[:, dim + k, :].astype(np.float64) + 8388608.0) * s + o).astype(np.float32)
    return refs, nc, lo, hi


@pytest.mark.parametrize("dim", [2, 3])
def test_quantised_boxes_contain_their_subtrees(dim):
    if dim == 3:
        v, f = W.icosphere(4, amplitude=0.3, seed=5)
    else:
        v, f = W.star_polyline(3000, seed=5)
    s = _host(v, f, dim)
    words = s.ref_array(L.ARRAY_WIDE_NODES)
    refs, nc, lo, hi = _decode_wide(words, dim)
    P = s.ref_array(L.ARRAY_PRIMITIVES).reshape(-1, dim * dim + 1)
    verts = P[:, :dim * dim].reshape(-1, dim, dim)
    eps = np.float32(np.finfo(np.float32).eps)
    plo, phi = verts.min(axis=1) - eps, verts.max(axis=1) + eps
    N = _nodes(s)
    leaf_len = {int(N[i, 2 * dim]): int(N[i, 2 * dim + 2]) for i in range(len(N)) if N[i, 2 * dim + 2] > 0}

    def prim_range(ref):
        if ref < 0 and (ref & 0x40000000) == 0:  # a run child: first | count << 24
            first, cnt = ref & 0xffffff, (ref >> 24) & 0x3f
            assert 1 <= cnt <= 6
            return [(first, first + cnt)]
        if ref < 0:
            o = ~ref
            return [(o, o + leaf_len[o])]
        out = []
        for k in range(nc[ref]):
            out += prim_range(int(refs[ref, k]))
        return out

    used = np.concatenate([refs[i, :nc[i]] for i in range(refs.shape[0])]).astype(np.int64)
    assert ((used < 0) & ((used & 0x40000000) == 0)).any(), "no run children"
    for node in range(refs.shape[0]):
        for k in range(nc[node]):
            rng = prim_range(int(refs[node, k]))
            idx = np.concatenate([np.arange(a, b) for a, b in rng])
            assert (lo[node, k] <= plo[idx].min(axis=0)).all()
            assert (hi[node, k] >= phi[idx].max(axis=0)).all()
    assert s.info["wide_stack"] <= 96


def _decode_wide16(words, dim):
    """The 16-bit bounds records, decoded like the kernels (fma(2^23 + q, 2^e, origin))."""
    stride = 28 if dim == 3 else 20
    w = words.view(np.uint32).reshape(-1, stride)
    f = words.reshape(-1, stride)
    origin = f[:, :dim]
    meta = w[:, 3] if dim == 3 else w[:, 2]
    q = w[:, 4:].copy().view(np.uint16).reshape(-1, 2 * dim, 8).astype(np.float64)
    exps = np.stack([(meta >> (8 * k)) & 0xff for k in range(dim)], axis=1).astype(np.int32) - 127
    nc = (meta >> 24).astype(np.int32)
    scale = np.ldexp(1.0, exps)
    lo = np.empty((w.shape[0], 8, dim), np.float32)
    hi = np.empty_like(lo)
    for k in range(dim):
        s, o = scale[:, k:k + 1], origin[:, k:k + 1].astype(np.float64)
        lo[:, :, k] = ((q[:, k, :] + 8388608.0) * s + o).astype(np.float32)
        hi[:, :, k] = ((q[:, dim + k, :] + 8388608.0) * s + o).astype(np.float32)
    return nc, lo, hi


@pytest.mark.parametrize("dim", [2, 3])
def test_16bit_bounds_contain_the_8bit_nodes_children(dim):
    """The 16-bit bounds (build_wide = 2) describe the same children as the 8-bit nodes,
    each decoded box contains the child's exact box (outward rounding), and the finer
    grid leaves less slack around the exact boxes than the 8-bit one."""
    if dim == 3:
        v, f = W.icosphere(4, amplitude=0.3, seed=5)
    else:
        v, f = W.star_polyline(3000, seed=5)
    s = _host(v, f, dim, build_wide=2)
    refs, nc8, lo8, hi8 = _decode_wide(s.ref_array(L.ARRAY_WIDE_NODES), dim)
    nc16, lo16, hi16 = _decode_wide16(s.ref_array(L.ARRAY_WIDE16_BOUNDS), dim)
    assert np.array_equal(nc8, nc16)
    # exact child boxes: the primitives below each child
    P = s.ref_array(L.ARRAY_PRIMITIVES).reshape(-1, dim * dim + 1)
    verts = P[:, :dim * dim].reshape(-1, dim, dim)
    eps = np.float32(np.finfo(np.float32).eps)
    plo, phi = verts.min(axis=1) - eps, verts.max(axis=1) + eps
    N = _nodes(s)
    leaf_len = {int(N[i, 2 * dim]): int(N[i, 2 * dim + 2]) for i in range(len(N)) if N[i, 2 * dim + 2] > 0}

    def prim_range(ref):
        if ref < 0 and (ref & 0x40000000) == 0:  # a run child: first | count << 24
            first, cnt = ref & 0xffffff, (ref >> 24) & 0x3f
            assert 1 <= cnt <= 6
            return [(first, first + cnt)]
        if ref < 0:
            o = ~ref
            return [(o, o + leaf_len[o])]
        out = []
        for k in range(nc8[ref]):
            out += prim_range(int(refs[ref, k]))
        return out

    slack8 = slack16 = 0.0
    for node in range(refs.shape[0]):
        for k in range(nc8[node]):
            idx = np.concatenate([np.arange(a, b) for a, b in prim_range(int(refs[node, k]))])
            elo, ehi = plo[idx].min(axis=0), phi[idx].max(axis=0)
            assert (lo16[node, k] <= elo).all() and (hi16[node, k] >= ehi).all()
            slack8 += float(np.sum(elo - lo8[node, k]) + np.sum(hi8[node, k] - ehi))
            slack16 += float(np.sum(elo - lo16[node, k]) + np.sum(hi16[node, k] - ehi))
    assert slack16 < 0.05 * slack8, (slack16, slack8)


def test_invalid_inputs_are_rejected():
    v = np.zeros((3, 3), np.float32)
    with pytest.raises(L.GQError) as ei:
        Scene(v, np.array([[0, 1, 5]], np.int32), 3, device=None)
    assert ei.value.status == L.GQ_ERR_INVALID and "out of range" in str(ei.value)
    with pytest.raises(L.GQError):
        Scene(v, np.zeros((0, 3), np.int32), 3, device=None)
    with pytest.raises(ValueError):
        Scene(v, np.zeros((4, 4), np.int32), 3, device=None)


@pytest.mark.parametrize("bad", [np.nan, np.inf, -np.inf])
@pytest.mark.parametrize("dim", [2, 3])
def test_non_finite_vertices_are_rejected(dim, bad):
    if dim == 3:
        v, f = W.icosphere(1, seed=0)
    else:
        v, f = W.star_polyline(40, seed=0)
    v = v.copy()
    v[3, dim - 1] = bad
    with pytest.raises(L.GQError) as ei:
        Scene(v, f, dim, device=None)
    assert ei.value.status == L.GQ_ERR_INVALID and "finite" in str(ei.value)
