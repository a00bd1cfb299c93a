"""B200-native geometry queries: closest point, ray intersection and closest
silhouette on 2D polylines and 3D triangle meshes, with gQuery's Polyline/Mesh API.

The queries run as hand-written sm_100a CUDA kernels in ``lib/libgq.so``
(built by :func:`gquery_b200.build_lib.build`); trees come from the CPU SAH-BVH
and SNCH builders in the same library.
"""
import os

# CUDA maps streams onto this many hardware work queues (8 unless set before the CUDA
# context exists); streams that share a queue run their work in order.  The serving
# runtime drives 11 streams by default, so its short steps would otherwise queue behind
# long ones on a shared queue.  Effective only when set before CUDA is first used.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

from .scene import Scene  # noqa: E402
from .shapes import Mesh, Polyline  # noqa: E402
from . import records  # noqa: E402

__all__ = ["Scene", "Mesh", "Polyline", "records"]
