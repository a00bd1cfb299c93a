"""The 3D node bound never excludes a child holding a silhouette, on the pair and
silhouette records real host builds produce (tests/sil_node_check.cpp walks every
query's whole tree and tests every record below each excluded child), for displaced
icospheres at the origin, scaled and far from it, an open mesh, and query points
spread around them, near the surface and near the centre."""
import json
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from gquery_b200 import _lib as L
from gquery_b200 import workloads as W
from gquery_b200.scene import Scene

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    exe = tmp_path_factory.mktemp("silnode") / "sil_node_check"
    subprocess.run(["g++", "-O2", "-ffp-contract=off", "-I", str(ROOT / "gquery_b200" / "csrc"),
                    str(ROOT / "tests" / "sil_node_check.cpp"), "-o", str(exe)], check=True)
    return exe


def _queries(v, n, seed):
    rng = np.random.default_rng(seed)
    lo, hi = v.min(0), v.max(0)
    c, ext = 0.5 * (lo + hi), (hi - lo).max()
    box = c + rng.uniform(-1.0, 1.0, size=(n, 3)) * ext  # around the shape
    near = v[rng.integers(0, len(v), n)] + rng.standard_normal((n, 3)) * 1e-3 * ext  # near the surface
    centre = c + rng.standard_normal((n // 4, 3)) * 0.05 * ext  # inside, seeing the surface head-on
    return np.concatenate([box, near, centre]).astype(np.float32)


def _run(checker, tmp_path, v, f, n=300, seed=0):
    s = Scene(v, f, 3, device=None)
    pairs = s.ref_array(L.ARRAY_SNCH_PAIRS)
    sils = s.ref_array(L.ARRAY_SIL_RECORDS)
    assert pairs.size % 40 == 0 and sils.size % 16 == 0 and pairs.size > 0
    q = _queries(v, n, seed)
    paths = [tmp_path / "pairs.bin", tmp_path / "sils.bin", tmp_path / "q.bin"]
    for p, a in zip(paths, (pairs, sils, q)):
        np.ascontiguousarray(a, np.float32).tofile(p)
    bound = float(np.abs(v).max())
    r = subprocess.run([str(checker), *map(str, paths), repr(bound)], capture_output=True, text=True, timeout=600)
    return r.returncode, json.loads(r.stdout), r.stderr


@pytest.mark.parametrize("level,amp,scale,offset", [
    (5, 0.3, 1.0, 0.0),      # the silhouette workload's field, smaller
    (4, 0.15, 1.0, 0.0),
    (4, 0.3, 1e3, 0.0),      # large coordinates
    (4, 0.3, 1.0, 500.0),    # far from the origin
    (4, 0.3, 1e-3, 0.0),     # small coordinates
])
def test_node_bound_sound_on_real_trees(checker, tmp_path, level, amp, scale, offset):
    v, f = W.icosphere(level, amplitude=amp, seed=level)
    v = (v.astype(np.float64) * scale + offset).astype(np.float32)
    rc, res, err = _run(checker, tmp_path, v, f)
    assert rc == 0 and res["unsound"] == 0, (res, err)
    # the bound does prune on these meshes (the walk visits every node outside the excluded
    # subtrees, so this share understates the pruning), the cone form at least as much as
    # the delta form
    assert res["excluded"] > 0.1 * res["children"], res
    assert res["cone"] >= 0.99 * res["delta"], res


def test_node_bound_sound_on_open_mesh(checker, tmp_path):
    # half of an icosphere: boundary edges are silhouettes for every query, and the nodes
    # above them must never be skipped
    v, f = W.icosphere(4, amplitude=0.2, seed=7)
    cz = v[f].mean(1)[:, 2]
    f = f[cz > 0.0]
    rc, res, err = _run(checker, tmp_path, v, f)
    assert rc == 0 and res["unsound"] == 0, (res, err)
    assert res["excluded"] > 0, res
