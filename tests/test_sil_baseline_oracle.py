"""The oracle's closest_silhouette_baseline for polylines against a plain-Python
restatement of Polyline.configure_silhouette (polyline.py:44-122) and of the baseline
loop (polyline.py:212-223, silhouette_vertex.py:40-53), in FP32 with numpy, on small
open and closed polylines with collinear vertices."""
import numpy as np

import oracle

f32 = np.float32


def _norm(v):
    return v * (f32(1.0) / np.sqrt(f32(v[0] * v[0] + v[1] * v[1]), dtype=f32))


def _cross(a, b):
    return f32(a[0] * b[1]) - f32(a[1] * b[0])


def _python_baseline(v, e, x):
    nb = {}
    for a, b in e.tolist():
        nb.setdefault(a, [-1, a, -1])
        nb.setdefault(b, [-1, b, -1])
        nb[a][2] = b
        nb[b][0] = a
    sils = []
    for i, key in enumerate(nb):
        p, c, n = nb[key]
        if p == -1 or n == -1:
            continue
        e1, e2 = _norm(v[c] - v[p]), _norm(v[n] - v[c])
        if abs(f32(e1[0] * e2[0]) + f32(e1[1] * e2[1])) < f32(1.0 - 1e-5):
            sils.append((v[p], v[c], v[n], i))
    out = []
    for q in x:
        best, d_min = None, np.inf
        for a, b, c, i in sils:
            w = q - b
            d = np.sqrt(f32(w[0] * w[0] + w[1] * w[1]), dtype=f32)
            if d < d_min and _cross(b - a, q - a) * _cross(c - b, q - b) < 0:
                best, d_min = i, d
        out.append((best is not None, -1 if best is None else best, d_min if best is not None else 0.0))
    return out


def test_polyline_baseline_matches_python_restatement():
    rng = np.random.default_rng(0)
    t = np.linspace(0, 2 * np.pi, 40, endpoint=False)
    closed = np.stack([np.cos(t), np.sin(t) * 0.5], 1).astype(f32)
    closed[5] = 0.5 * (closed[4] + closed[6])                   # a collinear vertex
    e_closed = np.stack([np.arange(40), (np.arange(40) + 1) % 40], 1)
    opened = rng.uniform(-1, 1, (15, 2)).astype(f32)
    e_open = np.stack([np.arange(14), np.arange(1, 15)], 1)      # open: both ends have one neighbour
    for v, e in ((closed, e_closed), (opened, e_open)):
        x = rng.uniform(-2, 2, (300, 2)).astype(f32)
        got = oracle.closest_silhouette_brute(2, x, vertices=v, indices=e.astype(np.int32))
        ref = _python_baseline(v, e, x)
        assert np.array_equal(got["valid"], [r[0] for r in ref])
        live = got["valid"]
        assert np.array_equal(got["prim_id"][live], np.array([r[1] for r in ref])[live])
        # the oracle's distance uses the same FP32 operations, the restatement numpy's
        assert np.allclose(got["d"][live], np.array([r[2] for r in ref])[live], rtol=1e-6)
