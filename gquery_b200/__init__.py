"""B200-native geometry queries: closest point, ray intersection and closest
silhouette on 2D polylines and 3D triangle meshes, with gQuery's Polyline/Mesh API.

The queries run as hand-written sm_100a CUDA kernels in ``lib/libgq.so``
(built by :func:`gquery_b200.build_lib.build`); trees come from the CPU SAH-BVH
and SNCH builders in the same library.
"""
from .scene import Scene
from .shapes import Mesh, Polyline
from . import records

__all__ = ["Scene", "Mesh", "Polyline", "records"]
