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


_HDR = "<8sii qq 6i qqq 4i 6f ff 6Q"  # the scene file header (176 bytes)


def _layout(raw: bytes):
    import struct
    f = struct.unpack_from(_HDR, raw, 0)
    dim, nv, np_ = f[2], f[3], f[4]
    sizes = f[-6:]
    off = struct.calcsize(_HDR) + nv * dim * 4 + np_ * dim * 4
    starts = []
    for s in sizes:
        starts.append(off)
        off += s
    return dim, np_, starts, sizes  # arrays: pairs, prims, spheres, wide nodes, SNCH pairs, silhouettes


def _patch(raw: bytes, at: int, value: int) -> bytes:
    import struct
    b = bytearray(raw)
    struct.pack_into("<i", b, at, value)
    return bytes(b)


def test_load_rejects_corrupt_trees(tmp_path):
    """A saved scene whose arrays disagree with each other is refused on the host before
    anything reaches the device: the kernels follow its references unchecked."""
    import struct
    v, f = W.icosphere(3, amplitude=0.2, seed=9)
    a = Scene(v, f, 3, device=0, build_snch=True)
    good = tmp_path / "good.gqs"
    a.save(good)
    raw = good.read_bytes()
    dim, np_, st, sz = _layout(raw)
    assert dim == 3 and sz[0] >= 64 and sz[3] >= 96 and sz[4] >= 160
    ref_l0 = struct.unpack_from("<i", raw, st[0] + 48)[0]
    cases = {
        "pair child past the pairs": _patch(raw, st[0] + 48, sz[0] // 64 + 3),
        "leaf past the primitives": _patch(raw, st[0] + 52, ~(np_ + 5)),
        "a node with two parents": _patch(raw, st[0] + 52, ref_l0) if ref_l0 >= 0 else None,
        "last primitive ends no leaf": _patch(raw, st[1] + (np_ - 1) * 48 + 40, 0),
        "wide node with nine children": _patch(raw, st[3] + 12, (struct.unpack_from("<I", raw, st[3] + 12)[0] & 0xffffff) | (9 << 24)),
        "SNCH child past the pairs": _patch(raw, st[4] + 88, sz[4] // 160 + 1),
    }
    for name, data in cases.items():
        if data is None:
            continue
        p = tmp_path / "bad.gqs"
        p.write_bytes(data)
        with pytest.raises(L.GQError, match="corrupt") as ei:
            Scene.load(p)
        assert ei.value.status == L.GQ_ERR_INVALID, name
    b = Scene.load(good)  # the file itself stays loadable
    q = W.uniform_points(4000, 3, seed=10)
    assert_bitwise(to_np(b.closest_point(q, variant="exact")), to_np(a.closest_point(q, variant="exact")),
                   ["valid", "p", "d", "prim_id"], "good file ")


def test_device_built_scene_round_trip(tmp_path):
    """Device-built trees number their nodes in the order of the sorted keys (a child may
    precede its parent); the load check accepts them."""
    v, f = W.icosphere(4, amplitude=0.2, seed=11)
    a = Scene(v, f, 3, device=0, build_snch=True, gpu_build=True)
    p = tmp_path / "gpu.gqs"
    a.save(p)
    b = Scene.load(p)
    q = W.uniform_points(8000, 3, seed=12)
    for variant in ("exact", "auto"):
        assert_bitwise(to_np(b.closest_point(q, variant=variant)), to_np(a.closest_point(q, variant=variant)),
                       ["valid", "p", "d", "prim_id"], f"cp {variant} ")
        assert_bitwise(to_np(b.closest_silhouette(q, variant=variant)),
                       to_np(a.closest_silhouette(q, variant=variant)), ["valid", "p", "d", "prim_id"], "sil ")
    assert b.device_error() == 0
