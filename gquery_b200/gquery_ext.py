"""Builder bindings under the names of gQuery's nanobind module ``gquery_ext``
(src/gquery.cpp:181-250), so scripts that build trees and read the flat float
arrays keep working.  The trees come from the same C++ builder as the GPU scenes.

    BVH(vertices [V, 2], indices [E, 2]).node_data()      -> float32, stride 7
    BVH3D(...).node_data() / primitive_data()             -> stride 9 / 10
    SNCH(...).node_data() / silhouette_data()             -> stride 13 / 10
    SNCH3D(...).node_data() / silhouette_data()           -> stride 16 / 19
    build_flat_silhouette_edges(vertices, indices)        -> stride 19
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .scene import Scene, _host_prims


class SceneArrays:
    """Reference arrays of a built scene (host copies)."""

    def __init__(self, scene: Scene, snch: bool):
        self._scene = scene
        self._snch = snch

    def node_data(self) -> np.ndarray:
        return self._scene.ref_array(L.ARRAY_SNCH_NODES if self._snch else L.ARRAY_BVH_NODES)

    def primitive_data(self) -> np.ndarray:
        return self._scene.ref_array(L.ARRAY_PRIMITIVES)

    def silhouette_data(self) -> np.ndarray:
        if not self._snch:
            raise AttributeError("silhouette_data belongs to SNCH objects")
        return self._scene.ref_array(L.ARRAY_SILHOUETTES)

    def raw_silhouette_data(self) -> np.ndarray:
        if not self._snch:
            raise AttributeError("raw_silhouette_data belongs to SNCH objects")
        return self._scene.ref_array(L.ARRAY_RAW_SILHOUETTES)


class _Builder(SceneArrays):
    dim = 0
    snch = False

    def __init__(self, vertices, indices, max_prims_in_node: int = 10):
        scene = Scene(vertices, indices, self.dim, device=None, build_snch=self.snch, build_wide=False,
                      max_prims_in_node=max_prims_in_node)
        super().__init__(scene, self.snch)


class BVH(_Builder):  # gquery.cpp:181-190
    dim = 2


class BVH3D(_Builder):  # gquery.cpp:193-202
    dim = 3


class SNCH(_Builder):  # gquery.cpp:226-235
    dim = 2
    snch = True


class SNCH3D(_Builder):  # gquery.cpp:238-247
    dim = 3
    snch = True


def build_flat_silhouette_edges(vertices, indices) -> np.ndarray:  # gquery.cpp:250
    v, f = _host_prims(vertices, indices, 3)
    n = C.c_int64()
    L.check(L.lib().gq_flat_silhouette_edges(v.ctypes.data, v.shape[0], f.ctypes.data, f.shape[0], None, 0,
                                             C.byref(n)))
    out = np.empty(n.value, np.float32)
    L.check(L.lib().gq_flat_silhouette_edges(v.ctypes.data, v.shape[0], f.ctypes.data, f.shape[0],
                                             out.ctypes.data, n.value, C.byref(n)))
    return out


def build_flat_silhouette_edges_device(vertices, indices, *, device: int = 0):
    """build_flat_silhouette_edges on the GPU: device torch tensors in ([V, 3] float32,
    [F, 3] int32, or anything torch can move there), a device float32 tensor out with
    the same values and order as the host function."""
    import torch
    dev = torch.device("cuda", device)
    v = torch.as_tensor(vertices).to(dev, torch.float32).contiguous()
    f = torch.as_tensor(indices).to(dev, torch.int32).contiguous()
    if v.dim() != 2 or f.dim() != 2:
        raise ValueError("vertices and indices must be 2-D")
    if v.shape[1] != 3 and v.shape[0] == 3:
        v = v.t().contiguous()
    if f.shape[1] != 3 and f.shape[0] == 3:
        f = f.t().contiguous()
    stream = torch.cuda.current_stream(dev).cuda_stream
    n = C.c_int64()
    L.check(L.lib().gq_flat_silhouette_edges_device(v.data_ptr(), v.shape[0], f.data_ptr(), f.shape[0], None, 0,
                                                    C.byref(n), device, stream))
    out = torch.empty(n.value, dtype=torch.float32, device=dev)
    L.check(L.lib().gq_flat_silhouette_edges_device(v.data_ptr(), v.shape[0], f.data_ptr(), f.shape[0],
                                                    out.data_ptr(), n.value, C.byref(n), device, stream))
    return out
