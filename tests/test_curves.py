"""The query-order keys (csrc/device/curves.cuh), built for the host by tests/curve_check.cpp:
on aligned blocks of grid cells (3D: 1024 cells per axis, 2D: 32768) the Hilbert indices
form one contiguous range, are distinct and step between face-adjacent cells only; the
top level of the 2D curve puts its four quadrants in the four quarters of the range; and
the Morton code, run through the same check as a control, fails it."""
import json
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def report(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    exe = tmp_path_factory.mktemp("curves") / "curve_check"
    subprocess.run(["g++", "-O2", "-Wno-unknown-pragmas", "-I", str(ROOT / "gquery_b200" / "csrc"),
                    str(ROOT / "tests" / "curve_check.cpp"), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    return json.loads(out)


def test_hilbert_blocks_3d(report):
    assert report["blocks3"] == 88
    assert (report["bad_range3"], report["bad_step3"], report["bad_unique3"]) == (0, 0, 0), report


def test_hilbert_blocks_2d(report):
    assert report["blocks2"] == 48
    assert (report["bad_range2"], report["bad_step2"], report["bad_unique2"]) == (0, 0, 0), report
    assert report["quarters2"] == 0b1111


def test_the_check_rejects_a_morton_order(report):
    assert report["morton_bad_step3"] > 0
