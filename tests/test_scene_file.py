"""Scene files: a loaded scene answers exactly like the scene it was saved from, and its
reference arrays (rebuilt on first use) are the same."""
import numpy as np
import pytest

from gquery_b200 import _lib as L
from gquery_b200 import workloads as W
from gquery_b200.scene import Scene
from parity import assert_bitwise, to_np

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dim", [2, 3])
def test_save_load_round_trip(dim, tmp_path):
    if dim == 2:
        v, f = W.star_polyline(3000, seed=4)
    else:
        v, f = W.icosphere(4, amplitude=0.2, seed=6)
    a = Scene(v, f, dim, device=0, build_snch=True)
    path = tmp_path / f"scene{dim}.gqs"
    a.save(path)
    b = Scene.load(path, device=0)
    for k in ("dim", "n_prims", "n_nodes", "n_wide_nodes", "n_silhouettes", "max_depth", "exact_stack", "wide_stack"):
        assert a.info[k] == b.info[k], k
    q = W.uniform_points(20000, dim, seed=7)
    o, d = W.rays(20000, dim, seed=8)
    for variant in ("exact", "auto"):
        assert_bitwise(to_np(b.closest_point(q, variant=variant)), to_np(a.closest_point(q, variant=variant)),
                       ["valid", "p", "d", "prim_id"], f"cp {variant} ")
        assert_bitwise(to_np(b.intersect(o, d, variant=variant)), to_np(a.intersect(o, d, variant=variant)),
                       ["valid", "p", "d", "prim_id"], f"ray {variant} ")
        assert_bitwise(to_np(b.closest_silhouette(q, variant=variant)),
                       to_np(a.closest_silhouette(q, variant=variant)), ["valid", "p", "d", "prim_id"], "sil ")
    for which in (L.ARRAY_BVH_NODES, L.ARRAY_PRIMITIVES, L.ARRAY_SNCH_NODES, L.ARRAY_SILHOUETTES):
        assert np.array_equal(a.ref_array(which).view(np.uint32), b.ref_array(which).view(np.uint32)), which
    assert b.device_error() == 0


def test_load_rejects_other_files(tmp_path):
    p = tmp_path / "not_a_scene.bin"
    p.write_bytes(b"hello world" * 10)
    with pytest.raises(L.GQError, match="not a saved scene"):
        Scene.load(p)
    with pytest.raises(L.GQError, match="cannot open"):
        Scene.load(tmp_path / "missing.gqs")
    v, f = W.icosphere(1)
    with pytest.raises(L.GQError, match="device copy"):
        Scene(v, f, 3, device=None).save(tmp_path / "x.gqs")
