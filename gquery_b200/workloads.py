"""Seeded synthetic scenes and queries with the shapes, sizes and value distributions of
the benchmark configurations (no datasets are needed or used).

    star_polyline    closed star polygon, r = 1 + 0.3 sin 7θ + 0.05 N(0,1)
    icosphere        subdivided icosahedron (20 * 4^level faces), optionally displaced
                     radially by 1 + a * sum_{k=1..4} sin(k (3x + 5y + 7z) + phi_k)
    uniform_points   U[lo, hi]^D queries
    sphere_dirs      uniform directions on S^1 / S^2 (normalised Gaussians)
"""
from __future__ import annotations

import math

import numpy as np


def star_polyline(n: int = 4096, seed: int = 0):
    rng = np.random.default_rng(seed)
    theta = 2.0 * np.pi * np.arange(n) / n
    r = 1.0 + 0.3 * np.sin(7.0 * theta) + 0.05 * rng.standard_normal(n)
    v = np.stack([r * np.cos(theta), r * np.sin(theta)], axis=1).astype(np.float32)
    e = np.stack([np.arange(n), (np.arange(n) + 1) % n], axis=1).astype(np.int32)
    return v, e


_ICO_FACES = np.array([
    (0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6),
    (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10),
    (8, 6, 7), (9, 8, 1)], dtype=np.int64)


def icosphere(level: int, amplitude: float = 0.0, seed: int = 0):
    """Unit icosphere with 20 * 4^level faces; returns (float32 [V,3], int32 [F,3])."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = np.array([(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
                  (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)], dtype=np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = _ICO_FACES.copy()
    for _ in range(level):
        nv, nf = v.shape[0], f.shape[0]
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]], axis=0)
        lo, hi = np.minimum(e[:, 0], e[:, 1]), np.maximum(e[:, 0], e[:, 1])
        key = lo * nv + hi
        uniq, inv = np.unique(key, return_inverse=True)
        ua, ub = uniq // nv, uniq % nv
        mid = v[ua] + v[ub]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        v = np.concatenate([v, mid], axis=0)
        m = nv + inv
        ab, bc, ca = m[:nf], m[nf:2 * nf], m[2 * nf:]
        a, b, c = f[:, 0], f[:, 1], f[:, 2]
        f = np.concatenate([np.stack([a, ab, ca], 1), np.stack([b, bc, ab], 1), np.stack([c, ca, bc], 1),
                            np.stack([ab, bc, ca], 1)], axis=0)
    if amplitude:
        rng = np.random.default_rng(seed)
        phi = rng.uniform(0.0, 2.0 * np.pi, size=4)
        s = 3.0 * v[:, 0] + 5.0 * v[:, 1] + 7.0 * v[:, 2]
        r = 1.0 + amplitude * sum(np.sin(k * s + phi[k - 1]) for k in range(1, 5))
        v = v * r[:, None]
    return v.astype(np.float32), f.astype(np.int32)


def uniform_points(n: int, dim: int, lo: float = -2.0, hi: float = 2.0, seed: int = 1) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.uniform(lo, hi, size=(n, dim)).astype(np.float32)


def sphere_dirs(n: int, dim: int, seed: int = 2) -> np.ndarray:
    rng = np.random.default_rng(seed)
    d = rng.standard_normal((n, dim))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return d.astype(np.float32)


def rays(n: int, dim: int, seed: int = 2):
    """Origins U[-2,2]^D and uniform directions, from one seeded stream."""
    rng = np.random.default_rng(seed)
    o = rng.uniform(-2.0, 2.0, size=(n, dim)).astype(np.float32)
    d = rng.standard_normal((n, dim))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return o, d.astype(np.float32)


# ---- benchmark configurations -------------------------------------------------

def config0(n_queries: int = 1 << 20):
    """2D closest point: 4,096-vertex star, 1,048,576 queries U[-2,2]^2."""
    v, e = star_polyline(4096, seed=0)
    return v, e, uniform_points(n_queries, 2, seed=1)


def config1_mesh():
    """Icosphere level 8 (1,310,720 triangles) displaced with amplitude 0.15."""
    return icosphere(8, amplitude=0.15, seed=0)


def config2_mesh():
    """Icosphere level 7 (327,680 triangles) displaced with amplitude 0.3."""
    return icosphere(7, amplitude=0.3, seed=0)


def config3_scenes(n_scenes: int = 512, lo: int = 64, hi: int = 262144):
    """Segment counts log-uniform in [lo, hi], one star polyline per scene (seed = scene id)."""
    out = []
    for sid in range(n_scenes):
        rng = np.random.default_rng(sid)
        m = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
        out.append(star_polyline(m, seed=sid))
    return out


def config3_queries(scenes, n_total: int = 1 << 24, mix=(0.5, 0.3, 0.2), seed: int = 7):
    """Per-scene query counts proportional to segment count (summing to n_total), each
    scene's queries uniform in its bounding box scaled 2x about its centre, split
    closest point / ray / silhouette by `mix` (rays: directions uniform on S^1).

    Returns {"cp": (ids, pts), "ray": (ids, origins, dirs), "sil": (ids, pts)} with
    int32 [n] scene ids and float32 [n, 2] arrays, grouped by scene."""
    rng = np.random.default_rng(seed)
    m = np.array([e.shape[0] for _, e in scenes], dtype=np.float64)
    counts = np.floor(n_total * m / m.sum()).astype(np.int64)
    counts[np.argsort(-m)[: n_total - counts.sum()]] += 1  # hand out the remainder to the largest scenes
    parts = {"cp": [], "ray": [], "sil": []}
    for sid, ((v, _), c) in enumerate(zip(scenes, counts)):
        lo, hi = v.min(axis=0).astype(np.float64), v.max(axis=0).astype(np.float64)
        mid, half = 0.5 * (lo + hi), 0.5 * (hi - lo)
        n_cp = int(round(c * mix[0]))
        n_ray = int(round(c * mix[1]))
        n_sil = int(c) - n_cp - n_ray
        for kind, k in (("cp", n_cp), ("ray", n_ray), ("sil", n_sil)):
            pts = (mid + rng.uniform(-2.0, 2.0, size=(k, 2)) * half).astype(np.float32)
            ids = np.full(k, sid, np.int32)
            if kind == "ray":
                a = rng.uniform(0.0, 2.0 * np.pi, size=k)
                dirs = np.stack([np.cos(a), np.sin(a)], axis=1).astype(np.float32)
                parts[kind].append((ids, pts, dirs))
            else:
                parts[kind].append((ids, pts))
    return {k: tuple(np.concatenate(col) for col in zip(*v)) for k, v in parts.items()}


def config4_levels(n_scenes: int = 64, lo: int = 4, hi: int = 8, seed: int = 11):
    """Subdivision level of each served scene: uniform over lo..hi, seeded."""
    rng = np.random.default_rng(seed)
    return [int(x) for x in rng.integers(lo, hi + 1, size=n_scenes)]


def config4_scene(sid: int, level: int):
    """Served scene `sid`: icosphere of `level` displaced with amplitude 0.15 (seed = 1000 + sid)."""
    return icosphere(level, amplitude=0.15, seed=1000 + sid)
