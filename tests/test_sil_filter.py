"""The silhouette-edge pre-test never excludes an edge the reference's test calls a
silhouette (random, nearly coplanar, sliver, zero-length, far and on-edge cases), and
without its margin it would: the cases reach the rounding boundary the margin covers.
The node bound never excludes a patch of edges (smooth, rough, flat or steep height
fields and spherical caps, whose records come in either orientation) that holds a
silhouette for the query."""
import json
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    exe = tmp_path_factory.mktemp("silf") / "sil_filter_check"
    subprocess.run(["g++", "-O2", "-ffp-contract=off", "-I", str(ROOT / "gquery_b200" / "csrc"),
                    str(ROOT / "tests" / "sil_filter_check.cpp"), "-o", str(exe)], check=True)
    return exe


def _run(exe, n, scale):
    p = subprocess.run([str(exe), str(n), str(scale)], capture_output=True, text=True, timeout=300)
    return p.returncode, json.loads(p.stdout)


def test_pre_test_is_sound(checker):
    rc, res = _run(checker, 400000, 1.0)
    assert rc == 0, res
    assert all(r["unsound"] == 0 for r in res.values()), res
    # it does exclude edges (otherwise it would be useless)
    assert res["generic"]["excluded"] > 0.3 * res["generic"]["cases"]
    # degenerate faces never use it
    assert res["zero_length"]["usable"] == 0
    # the node bound skips patches, and with mixed record orientations too
    for k in ("node_smooth", "node_rough", "node_flat"):
        assert res[k]["excluded"] > 0.2 * res[k]["cases"], (k, res[k])
    # the cone form is never wider than the delta form (rounding aside) ...
    for k in ("node_smooth", "node_rough", "node_flat", "node_cap", "node_steep"):
        assert res[k]["cone"] >= 0.999 * res[k]["delta"], (k, res[k])
    assert res["node_cap"]["cone"] > 0.3 * res["node_cap"]["cases"], res["node_cap"]
    # ... and skips patches whose normals spread 60 to 85 degrees when they are seen
    # head-on, where the delta form stops near 60
    w = res["node_steep"]
    assert w["cone"] > w["delta"] + 0.02 * w["cases"], w


def test_margin_is_needed(checker):
    rc, res = _run(checker, 400000, 0.0)
    assert rc == 1
    assert sum(r["unsound"] for r in res.values()) > 0
