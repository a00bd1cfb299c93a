"""Device-resident scene: the CPU SAH-BVH / SNCH build, the flattening pass and the
query entry points of libgq.so, with torch tensors in and out.
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Optional, Sequence, Union

import numpy as np
import torch

from . import _lib as L
from . import records as R

ArrayLike = Union[torch.Tensor, np.ndarray, Sequence]

VARIANTS = {"exact": L.VARIANT_EXACT, "wide8": L.VARIANT_WIDE8, "auto": L.VARIANT_AUTO,
            "coherent": L.VARIANT_COHERENT, "warp": L.VARIANT_WARP, "wide16": L.VARIANT_WIDE16}
KINDS = {"cp": L.KIND_CLOSEST_POINT, "ray": L.KIND_INTERSECT, "sil": L.KIND_SILHOUETTE}
VARIANT_NAMES = {v: k for k, v in VARIANTS.items()}


def _as_tensor(x) -> torch.Tensor:
    if isinstance(x, torch.Tensor):
        return x
    if hasattr(x, "__dlpack__") and not isinstance(x, np.ndarray):  # DrJit and other DLPack producers
        return torch.from_dlpack(x)
    return torch.as_tensor(np.asarray(x))


def points_layout(t: torch.Tensor, dim: int):
    """Returns (tensor, n, comp_stride, elem_stride) for a [D, n] (SoA, the reference's
    Array2/Array3 layout) or [n, D] (AoS) float32 tensor, without copying."""
    if t.dim() == 1:
        if t.shape[0] != dim:
            raise ValueError(f"expected {dim} components, got shape {tuple(t.shape)}")
        t = t.reshape(dim, 1)
    if t.dim() != 2:
        raise ValueError(f"expected a [{dim}, n] or [n, {dim}] array, got shape {tuple(t.shape)}")
    if t.shape[0] == dim:
        return t, t.shape[1], t.stride(0), t.stride(1)
    if t.shape[1] == dim:
        return t, t.shape[0], t.stride(1), t.stride(0)
    raise ValueError(f"expected a [{dim}, n] or [n, {dim}] array, got shape {tuple(t.shape)}")


def _host_prims(vertices, indices, dim):
    """Host float32 [nv, D] vertices and int32 [np, D] primitives from either layout."""
    v = _as_tensor(vertices).detach().to("cpu", torch.float32)
    f = _as_tensor(indices).detach().to("cpu", torch.int32)
    if v.dim() != 2 or f.dim() != 2:
        raise ValueError("vertices and indices must be 2-D arrays")
    if v.shape[1] != dim and v.shape[0] == dim:
        v = v.t()
    if f.shape[1] != dim and f.shape[0] == dim:
        f = f.t()
    if v.shape[1] != dim or f.shape[1] != dim:
        raise ValueError(f"expected [n, {dim}] or [{dim}, n] arrays")
    return np.ascontiguousarray(v.numpy()), np.ascontiguousarray(f.numpy())


def _ptr(t: Optional[torch.Tensor]) -> Optional[int]:
    return None if t is None else t.data_ptr()


def _stream_handle(stream) -> int:
    if stream is None:
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, torch.cuda.Stream):
        return stream.cuda_stream
    return int(stream)


class Scene:
    """One polyline (dim 2) or triangle mesh (dim 3) with its acceleration structures.

    ``device=None`` builds on the host only (reference arrays, no queries);
    ``gpu_build=True`` builds a linear BVH on the device in milliseconds (no reference
    arrays; answers equal to the host build's up to FP32 ties), its collapse into
    quantised 8-wide nodes (on the host, from the device-built pair records) and an SNCH
    on the same tree whose cones are taken from the geometry (mesh silhouette answers
    equal to closest_silhouette_baseline's, polyline ones to the host-built SNCH's, up
    to FP32 ties)."""

    def __init__(self, vertices: ArrayLike, indices: ArrayLike, dim: int, *, device: Optional[int] = 0,
                 build_snch: bool = True, build_wide: Union[bool, int] = True, max_prims_in_node: int = 10,
                 n_threads: int = 0, gpu_build: bool = False):
        if dim not in (2, 3):
            raise ValueError("dim must be 2 or 3")
        self.dim = dim
        v, f = _host_prims(vertices, indices, dim)
        self.vertices_host = v
        self.indices_host = f
        self.device = -1 if device is None else int(device)

        opts = L.BuildOpts(max_prims_in_node, n_threads, int(build_snch), int(build_wide), self.device,
                           int(gpu_build))
        h = C.c_void_p()
        build = L.lib().gq_scene_build_2d if dim == 2 else L.lib().gq_scene_build_3d
        L.check(build(v.ctypes.data, v.shape[0], f.ctypes.data, f.shape[0], C.byref(opts), C.byref(h)))
        self._h = h
        info = L.SceneInfo()
        L.check(L.lib().gq_scene_get_info(self._h, C.byref(info)))
        self.info = {k: (list(getattr(info, k)) if k.startswith("bbox") else getattr(info, k))
                     for k, _ in L.SceneInfo._fields_}
        self.has_snch = build_snch
        self.has_wide = bool(build_wide)
        self.has_wide16 = int(build_wide) >= 2 and not gpu_build
        self.torch_device = torch.device("cuda", self.device) if self.device >= 0 else None

    def save(self, path: str) -> None:
        """Writes the scene (geometry and flattened device arrays) for :meth:`load`."""
        L.check(L.lib().gq_scene_save(self._h, str(path).encode()))

    @classmethod
    def load(cls, path: str, *, device: int = 0) -> "Scene":
        """A scene saved by :meth:`save`, uploaded to `device` without rebuilding its
        trees (the reference arrays rebuild them on first use)."""
        h = C.c_void_p()
        L.check(L.lib().gq_scene_load(str(path).encode(), int(device), C.byref(h)))
        self = cls.__new__(cls)
        self._h = h
        info = L.SceneInfo()
        L.check(L.lib().gq_scene_get_info(self._h, C.byref(info)))
        self.info = {k: (list(getattr(info, k)) if k.startswith("bbox") else getattr(info, k))
                     for k, _ in L.SceneInfo._fields_}
        self.dim = self.info["dim"]
        self.vertices_host = self.indices_host = None
        self.device = int(device)
        self.has_snch = self.info["n_silhouettes"] > 0
        self.has_wide = self.info["n_wide_nodes"] > 0
        self.has_wide16 = False  # scene files keep the 8-bit nodes only
        self.torch_device = torch.device("cuda", self.device)
        return self

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            L.lib().gq_scene_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    # ---- reference float layouts (gquery_ext node_data() etc.) ----
    def ref_array(self, which: int) -> np.ndarray:
        n = C.c_int64()
        L.check(L.lib().gq_scene_ref_array(self._h, which, None, 0, C.byref(n)))
        out = np.empty(n.value, np.float32)
        L.check(L.lib().gq_scene_ref_array(self._h, which, out.ctypes.data, n.value, C.byref(n)))
        return out

    # ---- input staging ----
    def _points(self, x, name="points"):
        if self.torch_device is None:
            raise RuntimeError("scene was built without a device copy (device=None)")
        t = _as_tensor(x)
        if t.dtype != torch.float32 or t.device != self.torch_device:
            t = t.to(self.torch_device, torch.float32)
        t, n, cs, es = points_layout(t, self.dim)
        return t, n, L.Vecs(t.data_ptr(), cs, es)

    def _rmax(self, r_max, n):
        if r_max is None:
            return None
        if isinstance(r_max, (float, int)):
            if math.isinf(r_max) and r_max > 0:
                return None
            return torch.full((n,), float(r_max), dtype=torch.float32, device=self.torch_device)
        t = _as_tensor(r_max).to(self.torch_device, torch.float32).reshape(-1)
        if t.numel() == 1:
            if math.isinf(float(t.item())) and float(t.item()) > 0:
                return None
            t = t.expand(n)
        if t.numel() != n:
            raise ValueError("r_max must be a scalar or have one entry per query")
        return t.contiguous()

    def _opts(self, variant, sort, scratch, order=None):
        v = VARIANTS[variant] if isinstance(variant, str) else int(variant)
        o = None if order is None else order.data_ptr()
        if scratch is not None:
            return L.QueryOpts(v, int(sort), o, scratch.data_ptr(), scratch.numel() * scratch.element_size())
        return L.QueryOpts(v, int(sort), o, None, 0)

    def order(self, points, *, stream=None, scratch=None, out=None):
        """Permutation of the points along a Hilbert curve over twice the scene's box (int32
        [n] on the device)."""
        t, n, vq = self._points(points)
        perm = out if out is not None else self._alloc(n, torch.int32)
        sp, sb = (None, 0) if scratch is None else (scratch.data_ptr(), scratch.numel() * scratch.element_size())
        L.check(L.lib().gq_query_order(self._h, vq, n, perm.data_ptr(), sp, sb, _stream_handle(stream)))
        return perm

    def ray_order(self, origins, dirs, mode: int = 1, *, stream=None, scratch=None, out=None):
        """Permutation of rays (int32 [n] on the device) keyed by origin and direction:
        mode 0 the origins' point order, 1 direction octant then origin, 2 origin and direction
        interleaved."""
        t, n, vo = self._points(origins)
        td, n2, vd = self._points(dirs)
        if n2 != n:
            raise ValueError("origins and directions differ in length")
        perm = out if out is not None else self._alloc(n, torch.int32)
        sp, sb = (None, 0) if scratch is None else (scratch.data_ptr(), scratch.numel() * scratch.element_size())
        L.check(L.lib().gq_ray_order(self._h, vo, vd, n, int(mode), perm.data_ptr(), sp, sb, _stream_handle(stream)))
        return perm

    def get_tuning(self, kind: str) -> dict:
        t = L.Tuning()
        L.check(L.lib().gq_scene_get_tuning(self._h, KINDS[kind], C.byref(t)))
        d = {k: getattr(t, k) for k, _ in L.Tuning._fields_}
        d["variant"] = VARIANT_NAMES[d["variant"]]
        return d

    def set_tuning(self, kind: str, variant: str, packet: int = 0, sorted: int = 1, persist: int = 1,
                   budget: int = 32, block: int = 0, stack: int = 0) -> None:
        t = L.Tuning(VARIANTS[variant], packet, sorted, persist, budget, block, stack)
        L.check(L.lib().gq_scene_set_tuning(self._h, KINDS[kind], C.byref(t)))

    def scratch_bytes(self, n: int) -> int:
        return int(L.lib().gq_query_scratch_bytes(n))

    def _alloc(self, shape, dtype=torch.float32):
        return torch.empty(shape, dtype=dtype, device=self.torch_device)

    # ---- queries ----
    def closest_point(self, q, *, variant="auto", sort=True, stream=None, scratch=None, out=None, order=None):
        """closest_point_bvh (bvh.py:127-198 / bvh3d.py:108-174)."""
        t, n, vq = self._points(q)
        rec = out or self.alloc_cp(n)
        o = self.cp_out_struct(rec)
        opts = self._opts(variant, sort, scratch, order)
        L.check(L.lib().gq_closest_point(self._h, vq, n, C.byref(o), C.byref(opts), _stream_handle(stream)))
        return rec

    def alloc_cp(self, n):
        D = self.dim
        if D == 2:
            return R.ClosestPointRecord(self._alloc(n, torch.bool), self._alloc((2, n)), self._alloc((2, n)),
                                        self._alloc(n), self._alloc(n), self._alloc(n, torch.int32))
        return R.ClosestPointRecord3D(self._alloc(n, torch.bool), self._alloc((3, n)), self._alloc((3, n)),
                                      self._alloc((2, n)), self._alloc(n), self._alloc(n, torch.int32))

    def cp_out_struct(self, rec):
        t = rec.t if self.dim == 2 else rec.uv
        return L.CpOut(_ptr(rec.valid), _ptr(rec.p), _ptr(rec.n), _ptr(t), _ptr(rec.d), _ptr(rec.prim_id))

    def intersect(self, x, v, r_max=math.inf, *, variant="auto", sort=True, stream=None, scratch=None, out=None,
                  order=None):
        """intersect_bvh (bvh.py:200-276 / bvh3d.py:176-239)."""
        tx, n, vx = self._points(x)
        tv, n2, vv = self._points(v, "directions")
        if n2 != n:
            raise ValueError("origins and directions differ in length")
        rm = self._rmax(r_max, n)
        rec = out or self.alloc_ray(n)
        o = self.ray_out_struct(rec)
        opts = self._opts(variant, sort, scratch, order)
        L.check(L.lib().gq_intersect(self._h, vx, vv, _ptr(rm), n, C.byref(o), C.byref(opts),
                                     _stream_handle(stream)))
        return rec

    def alloc_ray(self, n):
        if self.dim == 2:
            return R.Intersection(self._alloc(n, torch.bool), self._alloc((2, n)), self._alloc((2, n)),
                                  self._alloc(n), self._alloc(n), self._alloc(n, torch.int32),
                                  self._alloc(n, torch.bool))
        return R.Intersection3D(self._alloc(n, torch.bool), self._alloc((3, n)), self._alloc((3, n)),
                                self._alloc((2, n)), self._alloc(n), self._alloc(n, torch.int32),
                                self._alloc(n, torch.bool))

    def ray_out_struct(self, rec):
        t = rec.t if self.dim == 2 else rec.uv
        return L.RayOut(_ptr(rec.valid), _ptr(rec.p), _ptr(rec.n), _ptr(t), _ptr(rec.d), _ptr(rec.prim_id),
                        _ptr(rec.on_boundary))

    def closest_silhouette(self, x, r_max=math.inf, *, variant="auto", sort=True, stream=None, scratch=None,
                           out=None, order=None):
        """closest_silhouette_snch (snch.py:106-164 / snch3d.py:143-203); variant "exact"
        (reference visit order), "coherent" (one traversal per warp of neighbouring
        queries) or "warp" (one query per warp); the last two give the same answers
        except at FP32 distance ties."""
        tx, n, vx = self._points(x)
        rm = self._rmax(r_max, n)
        rec = out or self.alloc_sil(n)
        o = L.SilOut(_ptr(rec.valid), _ptr(rec.p), _ptr(rec.d), _ptr(rec.prim_id))
        opts = self._opts(variant, sort, scratch, order)
        L.check(L.lib().gq_closest_silhouette(self._h, vx, _ptr(rm), n, C.byref(o), C.byref(opts),
                                              _stream_handle(stream)))
        return rec

    def alloc_sil(self, n):
        cls = R.ClosestSilhouettePointRecord if self.dim == 2 else R.ClosestSilhouettePointRecord3D
        return cls(self._alloc(n, torch.bool), self._alloc((self.dim, n)), self._alloc(n),
                   self._alloc(n, torch.int32))

    def closest_point_brute(self, q, *, stream=None):
        """closest_point_baseline (polyline.py:176-209, mesh.py closest_point_baseline)."""
        t, n, vq = self._points(q)
        rec = self.alloc_cp(n)
        o = self.cp_out_struct(rec)
        L.check(L.lib().gq_closest_point_brute(self._h, vq, n, C.byref(o), _stream_handle(stream)))
        return rec

    def intersect_brute(self, x, v, r_max=math.inf, *, stream=None):
        """intersect_baseline (polyline.py:138-169, mesh.py intersect_baseline)."""
        tx, n, vx = self._points(x)
        tv, _, vv = self._points(v)
        rm = self._rmax(r_max, n)
        rec = self.alloc_ray(n)
        o = self.ray_out_struct(rec)
        L.check(L.lib().gq_intersect_brute(self._h, vx, vv, _ptr(rm), n, C.byref(o), _stream_handle(stream)))
        return rec

    def closest_silhouette_brute(self, x, r_max=math.inf, *, stream=None):
        """closest_silhouette_baseline (polyline.py:212-223, mesh.py:124-135): every
        silhouette of the shape's list in order, the first strictly nearest kept."""
        tx, n, vx = self._points(x)
        rm = self._rmax(r_max, n)
        rec = self.alloc_sil(n)
        o = L.SilOut(_ptr(rec.valid), _ptr(rec.p), _ptr(rec.d), _ptr(rec.prim_id))
        L.check(L.lib().gq_closest_silhouette_brute(self._h, vx, _ptr(rm), n, C.byref(o), _stream_handle(stream)))
        return rec

    def brute_f64(self, kind: str, a, b=None, *, stream=None):
        """FP64 brute force, kind "cp" / "ray" / "sil": (distance, ray parameter or silhouette
        distance [float64, +inf when none], primitive or silhouette record id [int32])."""
        ta, n, va = self._points(a)
        vb = L.Vecs(None, 0, 0)
        if kind == "ray":
            tb, _, vb = self._points(b)
        d = torch.empty(n, dtype=torch.float64, device=self.torch_device)
        idx = torch.empty(n, dtype=torch.int32, device=self.torch_device)
        L.check(L.lib().gq_brute_f64(self._h, {"cp": 0, "ray": 1, "sil": 2}[kind], va, vb, n, d.data_ptr(), idx.data_ptr(),
                                     _stream_handle(stream)))
        return d, idx

    def set_stack_limit(self, entries: int) -> None:
        """Caps the traversal stacks at `entries` (0: the compiled sizes).  Queries whose
        walk needs more come back as misses and raise the stack bit of device_error()."""
        L.check(L.lib().gq_scene_set_stack_limit(self._h, int(entries)))

    def device_error(self, stream=None) -> int:
        v = C.c_int32()
        L.check(L.lib().gq_scene_device_error(self._h, _stream_handle(stream), C.byref(v)))
        return v.value
