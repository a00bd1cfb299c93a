"""Many scenes, all three query kinds, one launch per step (``gq_batch_*`` in libgq.so).

The reference answers one scene and one query kind per call (Mesh.closest_point_bvh,
mesh.py:120; Mesh.intersect_bvh, mesh.py:87; Mesh.closest_silhouette_snch,
mesh.py:138; and the Polyline counterparts).  A :class:`SceneBatch` holds device views
of many scenes of one dimension and answers a mixed step - closest points, rays and
silhouette queries, each tagged with its scene - in one persistent launch, with the
answers of the single-scene calls (closest points and silhouettes: ``coherent``; rays:
``wide8`` when every scene has wide nodes).  ``run`` allocates nothing on the
device beyond the output records, so a step with fixed shapes can be recorded in a CUDA
graph (:meth:`SceneBatch.capture`).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from typing import Optional, Sequence

import torch

from . import _lib as L
from .scene import Scene, _ptr, _stream_handle, points_layout

SKIP = -1  # scene index of a padding slot: skipped, its outputs left untouched


@dataclass
class BatchResult:
    cp: object = None
    ray: object = None
    sil: object = None


class SceneBatch:
    """Device views of ``scenes`` (same dimension and device; they must stay alive) and a
    fixed scratch for up to ``max_queries`` queries of each kind.

    ``cp_variant`` / ``sil_variant``: "coherent" (warp-coherent traversal) or "exact"
    (reference visit order, one lane per query); silhouettes also "warp" (one query per
    warp, for sparse queries).  ``ray_variant``: "wide8" or "exact"."""

    def __init__(self, scenes: Sequence[Scene], max_queries: int, *, cp_variant: str = "coherent",
                 ray_variant: str = "wide8", sil_variant: str = "coherent"):
        if not scenes:
            raise ValueError("a batch needs at least one scene")
        if cp_variant not in ("coherent", "exact", "split") or ray_variant not in ("wide8", "exact") or \
                sil_variant not in ("coherent", "exact", "warp", "split"):
            raise ValueError("cp_variant: coherent|exact|split, ray_variant: wide8|exact, "
                             "sil_variant: coherent|exact|warp|split")
        self.scenes = list(scenes)
        self.dim = self.scenes[0].dim
        self.torch_device = self.scenes[0].torch_device
        self.max_queries = int(max_queries)
        flags = (L.BATCH_CP_EXACT if cp_variant == "exact" else L.BATCH_CP_SPLIT if cp_variant == "split" else 0) | \
            (L.BATCH_RAY_EXACT if ray_variant == "exact" else 0) | \
            (L.BATCH_SIL_EXACT if sil_variant == "exact" else L.BATCH_SIL_WARP if sil_variant == "warp" else
             L.BATCH_SIL_SPLIT if sil_variant == "split" else 0)
        arr = (C.c_void_p * len(self.scenes))(*[s.handle.value for s in self.scenes])
        h = C.c_void_p()
        L.check(L.lib().gq_batch_create(arr, len(self.scenes), self.max_queries, flags, C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            L.lib().gq_batch_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def device_bytes(self) -> int:
        return int(L.lib().gq_batch_device_bytes(self._h))

    # ---- staging ----
    def _vecs(self, x):
        t = x if isinstance(x, torch.Tensor) else torch.as_tensor(x)
        if t.dtype != torch.float32 or t.device != self.torch_device:
            t = t.to(self.torch_device, torch.float32)
        t, n, cs, es = points_layout(t, self.dim)
        return t, n, L.Vecs(t.data_ptr(), cs, es)

    def _ids(self, ids, n):
        t = ids if isinstance(ids, torch.Tensor) else torch.as_tensor(ids)
        if t.dtype != torch.int32 or t.device != self.torch_device:
            t = t.to(self.torch_device, torch.int32)
        t = t.reshape(-1).contiguous()
        if t.numel() != n:
            raise ValueError("one scene index per query")
        return t

    def _rmax(self, r_max, n):
        if r_max is None:
            return None
        if isinstance(r_max, (float, int)):
            if math.isinf(r_max) and r_max > 0:
                return None
            return torch.full((n,), float(r_max), dtype=torch.float32, device=self.torch_device)
        t = r_max.to(self.torch_device, torch.float32).reshape(-1).contiguous()
        if t.numel() != n:
            raise ValueError("r_max must be a scalar or have one entry per query")
        return t

    def alloc(self, n_cp: int = 0, n_ray: int = 0, n_sil: int = 0) -> BatchResult:
        s0 = self.scenes[0]
        return BatchResult(s0.alloc_cp(n_cp) if n_cp else None, s0.alloc_ray(n_ray) if n_ray else None,
                           s0.alloc_sil(n_sil) if n_sil else None)

    # ---- one step ----
    def run(self, cp=None, ray=None, sil=None, *, out: Optional[BatchResult] = None, stream=None) -> BatchResult:
        """cp = (points, scene_ids); ray = (origins, directions, scene_ids[, r_max]);
        sil = (points, scene_ids[, r_max]).  Points are [D, n] or [n, D] float32 device
        tensors, scene ids int32 [n] (``SKIP`` marks a padding slot)."""
        keep = []  # staged tensors must outlive the asynchronous launch
        qs = [None, None, None]
        ns = [0, 0, 0]
        if cp is not None:
            t, n, va = self._vecs(cp[0])
            ids = self._ids(cp[1], n)
            keep += [t, ids]
            qs[0] = L.BatchQueries(n, ids.data_ptr(), va, L.Vecs(None, 0, 0), None)
            ns[0] = n
        if ray is not None:
            tx, n, vx = self._vecs(ray[0])
            tv, n2, vv = self._vecs(ray[1])
            if n2 != n:
                raise ValueError("origins and directions differ in length")
            ids = self._ids(ray[2], n)
            rm = self._rmax(ray[3] if len(ray) > 3 else None, n)
            keep += [tx, tv, ids, rm]
            qs[1] = L.BatchQueries(n, ids.data_ptr(), vx, vv, _ptr(rm))
            ns[1] = n
        if sil is not None:
            t, n, va = self._vecs(sil[0])
            ids = self._ids(sil[1], n)
            rm = self._rmax(sil[2] if len(sil) > 2 else None, n)
            keep += [t, ids, rm]
            qs[2] = L.BatchQueries(n, ids.data_ptr(), va, L.Vecs(None, 0, 0), _ptr(rm))
            ns[2] = n
        res = out or self.alloc(*ns)
        s0 = self.scenes[0]
        co = s0.cp_out_struct(res.cp) if res.cp is not None else None
        ro = s0.ray_out_struct(res.ray) if res.ray is not None else None
        so = (L.SilOut(_ptr(res.sil.valid), _ptr(res.sil.p), _ptr(res.sil.d), _ptr(res.sil.prim_id))
              if res.sil is not None else None)

        def ref(x):
            return C.byref(x) if x is not None else None

        L.check(L.lib().gq_batch_run(self._h, ref(qs[0]), ref(co), ref(qs[1]), ref(ro), ref(qs[2]), ref(so),
                                     _stream_handle(stream)))
        self._keep = keep
        return res

    def capture(self, n_cp: int = 0, n_ray: int = 0, n_sil: int = 0) -> "BatchGraph":
        """Records one step of fixed sizes in a CUDA graph over static input tensors."""
        return BatchGraph(self, n_cp, n_ray, n_sil)

    def device_error(self, stream=None) -> int:
        v = C.c_int32()
        L.check(L.lib().gq_batch_device_error(self._h, _stream_handle(stream), C.byref(v)))
        return v.value


class BatchGraph:
    """A CUDA graph of one batch step with static inputs (``cp_points``, ``cp_scene``,
    ``ray_origin``, ``ray_dir``, ``ray_scene``, ``ray_rmax``, ``sil_points``,
    ``sil_scene``, ``sil_rmax``; points [D, n]) and static outputs (``out``).  Fill the
    inputs (unused slots: scene ``SKIP``), then :meth:`replay`."""

    def __init__(self, batch: SceneBatch, n_cp: int, n_ray: int, n_sil: int):
        if max(n_cp, n_ray, n_sil) > batch.max_queries:
            raise ValueError("graph sizes exceed the batch's max_queries")
        dev, D = batch.torch_device, batch.dim
        z = lambda *shape: torch.zeros(shape, dtype=torch.float32, device=dev)  # noqa: E731
        skip = lambda n: torch.full((n,), SKIP, dtype=torch.int32, device=dev)  # noqa: E731
        self.batch = batch
        self.sizes = (n_cp, n_ray, n_sil)
        self.cp_points, self.cp_scene = z(D, n_cp), skip(n_cp)
        self.ray_origin, self.ray_dir, self.ray_scene = z(D, n_ray), z(D, n_ray), skip(n_ray)
        self.ray_rmax = torch.full((n_ray,), math.inf, dtype=torch.float32, device=dev)
        self.sil_points, self.sil_scene = z(D, n_sil), skip(n_sil)
        self.sil_rmax = torch.full((n_sil,), math.inf, dtype=torch.float32, device=dev)
        self.out = batch.alloc(n_cp, n_ray, n_sil)
        if n_ray:
            self.ray_dir[0].fill_(1.0)
        # one eager step first: it caches the launch shapes outside the capture
        self._step()
        torch.cuda.current_stream(dev).synchronize()
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self._step()

    def _step(self):
        n_cp, n_ray, n_sil = self.sizes
        self.batch.run(cp=(self.cp_points, self.cp_scene) if n_cp else None,
                       ray=(self.ray_origin, self.ray_dir, self.ray_scene, self.ray_rmax) if n_ray else None,
                       sil=(self.sil_points, self.sil_scene, self.sil_rmax) if n_sil else None, out=self.out)

    def replay(self):
        self.graph.replay()
        return self.out
