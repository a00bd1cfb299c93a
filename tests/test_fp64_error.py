"""Error of the FP32 traversal against FP64 brute force for the query types the other
tests leave out: 2D rays and closest silhouettes (2D vertices, 3D edges).  The oracle's
FP32 traversal is the measured side (the exact GPU kernels equal it bit for bit); the
FP64 side is a numpy scan over every primitive or silhouette.  Closest points and 3D rays
are measured the same way in test_oracle_kat.py and test_gpu_parity.py."""
import numpy as np
import pytest

import oracle
from gquery_b200 import gquery_ext as gx
from gquery_b200 import workloads as W

ABS_TOL = 5e-7  # about 2 ulp of coordinates of magnitude 2


def _ray2d_fp64(v, e, o, d):
    """Nearest hit parameter t > 0 of each ray against every segment (inf: miss)."""
    a = v[e[:, 0]].astype(np.float64)[None]  # [1, E, 2]
    b = v[e[:, 1]].astype(np.float64)[None]
    o = o.astype(np.float64)[:, None]  # [N, 1, 2]
    d = d.astype(np.float64)[:, None]
    u = b - a
    den = d[..., 0] * u[..., 1] - d[..., 1] * u[..., 0]
    w = a - o
    with np.errstate(divide="ignore", invalid="ignore"):
        t = (w[..., 0] * u[..., 1] - w[..., 1] * u[..., 0]) / den
        s = (w[..., 0] * d[..., 1] - w[..., 1] * d[..., 0]) / den
    ok = (den != 0) & (t > 0) & (s >= 0) & (s <= 1)
    return np.where(ok, t, np.inf).min(axis=1)


def _sil2d_fp64(v, e, x):
    """Nearest silhouette vertex: a vertex b with both neighbours a, c (closed polyline)
    where cross(b - a, x - a) * cross(c - b, x - b) < 0."""
    nv = v.shape[0]
    prev = np.full(nv, -1)
    nxt = np.full(nv, -1)
    prev[e[:, 1]] = e[:, 0]
    nxt[e[:, 0]] = e[:, 1]
    keep = (prev >= 0) & (nxt >= 0)
    b = v[keep].astype(np.float64)[None]
    a = v[prev[keep]].astype(np.float64)[None]
    c = v[nxt[keep]].astype(np.float64)[None]
    xx = x.astype(np.float64)[:, None]

    def cross(p, q):
        return p[..., 0] * q[..., 1] - p[..., 1] * q[..., 0]
    sil = cross(b - a, xx - a) * cross(c - b, xx - b) < 0
    dist = np.linalg.norm(xx - b, axis=-1)
    return np.where(sil, dist, np.inf).min(axis=1)


def _sil3d_fp64(raw, x):
    """Nearest silhouette edge over the raw records (c, a, b, d; boundary edges always
    count): closest point q of [a, b], silhouette when (q - x) . n0 and (q - x) . n1
    differ in sign, n0 = cross(b - a, c - a), n1 = cross(d - a, b - a)."""
    r = raw.reshape(-1, 19).astype(np.float64)
    c, a, b, d = r[:, 0:3], r[:, 3:6], r[:, 6:9], r[:, 9:12]
    boundary = (r[:, 12].astype(np.float32).view(np.int32) == -1) | (r[:, 15].astype(np.float32).view(np.int32) == -1)
    n0 = np.cross(b - a, c - a)
    n1 = np.cross(d - a, b - a)
    u = b - a
    uu = np.maximum((u * u).sum(1), 1e-300)
    out = np.full(x.shape[0], np.inf)
    for i0 in range(0, x.shape[0], 256):
        xx = x[i0:i0 + 256].astype(np.float64)[:, None]
        t = np.clip(((xx - a[None]) * u[None]).sum(-1) / uu[None], 0.0, 1.0)
        q = a[None] + t[..., None] * u[None]
        w = q - xx
        sil = boundary[None] | ((w * n0[None]).sum(-1) * (w * n1[None]).sum(-1) < 0)
        out[i0:i0 + 256] = np.where(sil, np.linalg.norm(w, axis=-1), np.inf).min(axis=1)
    return out


def _raw_f32_view(raw):
    # the flat records hold int fields as float bit patterns: keep them as float32 bits
    return np.ascontiguousarray(raw, np.float32)


def test_ray2d_error_vs_fp64():
    v, e = W.star_polyline(1000, seed=6)
    b = gx.BVH(v, e)
    o, d = W.rays(3000, 2, seed=5)
    r = oracle.intersect(2, b.node_data(), b.primitive_data(), o, d)
    t64 = _ray2d_fp64(v, e, o, d)
    hit64 = np.isfinite(t64)
    # hit / miss differ only for rays grazing a segment end point
    assert (r["valid"] == hit64).mean() > 0.999
    both = r["valid"] & hit64
    err = np.abs(r["d"][both].astype(np.float64) - t64[both]) / np.maximum(t64[both], 1.0)
    assert err.max() < 4 * ABS_TOL, err.max()


def test_sil2d_error_vs_fp64():
    v, e = W.star_polyline(2000, seed=4)
    s = gx.SNCH(v, e)
    x = W.uniform_points(4000, 2, seed=8)
    r = oracle.closest_silhouette(2, s.node_data(), s.silhouette_data(), x)
    d64 = _sil2d_fp64(v, e, x)
    hit64 = np.isfinite(d64)
    assert (r["valid"] == hit64).mean() > 0.999
    both = r["valid"] & hit64
    err = np.abs(r["d"][both].astype(np.float64) - d64[both])
    # the silhouette condition flips within rounding of its sign for a few queries, which
    # then take the next silhouette; every other distance is within the FP32 rounding
    assert np.mean(err <= ABS_TOL) > 0.999, np.sort(err)[-5:]
    assert np.median(err) <= ABS_TOL


def test_sil3d_error_vs_fp64():
    v, f = W.icosphere(3, amplitude=0.3, seed=3)
    s = gx.SNCH3D(v, f)
    x = W.uniform_points(2000, 3, seed=12)
    r = oracle.closest_silhouette(3, s.node_data(), s.silhouette_data(), x)
    raw = _raw_f32_view(gx.build_flat_silhouette_edges(v, f))
    d64 = _sil3d_fp64(raw, x)
    hit64 = np.isfinite(d64)
    assert (r["valid"] == hit64).mean() > 0.999
    both = r["valid"] & hit64
    err = r["d"][both].astype(np.float64) - d64[both]
    # FP32 rounding, and the reference's cone test: it may skip the nearest silhouette
    # (its cones see one face normal and measure their radius from edge midpoints), so a
    # few queries end on a farther one (err > 0), never on a nearer one
    assert err.min() > -ABS_TOL, err.min()
    assert np.mean(np.abs(err) <= ABS_TOL) > 0.99, np.sort(err)[-5:]


# ---------------------------------------------------------------- the GPU FP64 silhouette scan

@pytest.mark.gpu
def test_gpu_fp64_silhouette_scan_matches_numpy():
    """gq_brute_f64 kind 2 (the FP64 silhouette reference the bench uses at full size)
    against the numpy FP64 scans above on the same raw silhouette lists."""
    from gquery_b200 import _lib as L
    from gquery_b200.scene import Scene
    v, e = W.star_polyline(2000, seed=4)
    s = Scene(v, e, 2, device=0)
    x = W.uniform_points(3000, 2, seed=8)
    d, ids = s.brute_f64("sil", x)
    d = d.cpu().numpy()
    d_np = _sil2d_fp64(v, e, x)
    assert np.array_equal(np.isinf(d), np.isinf(d_np))
    fin = np.isfinite(d_np)
    assert np.allclose(d[fin], d_np[fin], rtol=1e-12, atol=0)
    assert np.all(ids.cpu().numpy()[~fin] == -1)

    v3, f3 = W.icosphere(3, amplitude=0.3, seed=3)
    s3 = Scene(v3, f3, 3, device=0)
    x3 = W.uniform_points(3000, 3, seed=12)
    d3, _ = s3.brute_f64("sil", x3)
    d3 = d3.cpu().numpy()
    d3_np = _sil3d_fp64(_raw_f32_view(s3.ref_array(L.ARRAY_RAW_SILHOUETTES)), x3)
    assert np.array_equal(np.isinf(d3), np.isinf(d3_np))
    fin = np.isfinite(d3_np)
    assert np.allclose(d3[fin], d3_np[fin], rtol=1e-12, atol=0)
