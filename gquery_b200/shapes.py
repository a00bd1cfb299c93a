"""Drop-in ``Polyline`` / ``Mesh`` with gQuery's method names
(gquery/shapes/polyline.py:11-227, gquery/shapes/mesh.py:10-139).

Inputs: torch tensors (any device), numpy arrays, or DLPack producers such as DrJit
arrays, in the reference's component-major layout ``[D, n]`` or row-major ``[n, D]``.
Outputs: the records of :mod:`gquery_b200.records` holding CUDA tensors.
Every query runs on the GPU through libgq.so; there is no CPU path.
"""
from __future__ import annotations

import math

import torch

from . import gquery_ext
from .scene import Scene, _as_tensor


class _Shape:
    dim = 0

    def __init__(self, vertices, indices, *, device: int = 0, max_prims_in_node: int = 10,
                 build_wide: bool = True, sort_queries: bool = True, variant: str = "auto"):
        self.scene = Scene(vertices, indices, self.dim, device=device, build_snch=True, build_wide=build_wide,
                           max_prims_in_node=max_prims_in_node)
        self.sort_queries = sort_queries
        self.variant = variant
        dev = self.scene.torch_device
        self.vertices = torch.as_tensor(self.scene.vertices_host).t().contiguous().to(dev)  # [D, V]
        self.indices = torch.as_tensor(self.scene.indices_host).t().contiguous().to(dev)    # [D, P]
        self.bvh = gquery_ext.SceneArrays(self.scene, snch=False)
        self.snch = gquery_ext.SceneArrays(self.scene, snch=True)

    # ---- accelerated queries ----
    def closest_point_bvh(self, p):
        return self.scene.closest_point(p, variant=self.variant, sort=self.sort_queries)

    def intersect_bvh(self, p, v, r_max=math.inf):
        return self.scene.intersect(p, v, r_max, variant=self.variant, sort=self.sort_queries)

    def closest_silhouette_snch(self, x, r_max=math.inf):
        variant = self.variant if self.variant in ("exact", "coherent", "warp") else "auto"  # no wide silhouettes
        return self.scene.closest_silhouette(x, r_max, variant=variant, sort=self.sort_queries)

    # ---- brute-force scans (the reference's *_baseline methods) ----
    def closest_point_baseline(self, p):
        return self.scene.closest_point_brute(p)

    def intersect_baseline(self, p, v, r_max=math.inf):
        return self.scene.intersect_brute(p, v, r_max)

    def closest_silhouette_baseline(self, x, r_max=math.inf):
        return self.scene.closest_silhouette_brute(x, r_max)


class Polyline(_Shape):
    """2D polyline: ``Polyline(vertices [2, V] float32, indices [2, E] int32)`` (polyline.py:20)."""
    dim = 2

    def intersect(self, p, v, n=None, on_boundary=None, r_max=math.inf):
        """Ray cast from an optionally offset origin (polyline.py:124-130):
        origins flagged on_boundary move by -1e-5 * n before the brute-force scan."""
        p = _as_tensor(p).to(self.scene.torch_device, torch.float32)
        if n is not None and on_boundary is not None:
            n = _as_tensor(n).to(p.device, torch.float32)
            ob = _as_tensor(on_boundary).to(p.device, torch.bool).reshape(-1)
            # one flag per ray: along the last axis of [D, n] points, the first of [n, D]
            soa = p.dim() == 2 and p.shape[0] == self.dim and p.shape[1] == ob.numel()
            ob = ob[None, :] if soa else ob[:, None]
            p = torch.where(ob, p - 1e-5 * n, p)
        return self.intersect_baseline(p, v, r_max)


class Mesh(_Shape):
    """3D triangle mesh: ``Mesh(vertices [3, V] float32, indices [3, F] int32)`` (mesh.py:19)."""
    dim = 3
