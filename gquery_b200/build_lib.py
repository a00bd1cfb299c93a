"""Builds libgq.so in-tree (gquery_b200/lib/libgq.so) for sm_100a.

Host C++ (builders, flattening pass, C ABI) is compiled with g++ without
floating-point contraction; device code with nvcc for sm_100a with --fmad=false,
so that the fixed rounding rules of csrc/gq_fmath.h hold on both sides.
The CUDA runtime is linked statically.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
ROOT = PKG.parent
BUILD = ROOT / "_build" / "gq"
LIB = PKG / "lib" / "libgq.so"

HOST_SOURCES = ["host/scene_build.cpp", "host/flatten.cpp", "capi.cpp", "server.cpp"]
DEVICE_SOURCES = ["device/queries.cu", "device/traverse.cu", "device/packet.cu", "device/ray_group.cu",
                  "device/noalloc.cu", "device/batch.cu", "device/gpu_build.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _cuda_home() -> Path:
    for cand in (os.environ.get("CUDA_HOME"), "/usr/local/cuda"):
        if cand and (Path(cand) / "bin" / "nvcc").exists():
            return Path(cand)
    nvcc = shutil.which("nvcc")
    if nvcc:
        return Path(nvcc).resolve().parent.parent
    raise RuntimeError("nvcc not found (set CUDA_HOME)")


def _all_inputs():
    files = list(CSRC.rglob("*.cpp")) + list(CSRC.rglob("*.cu")) + list(CSRC.rglob("*.h")) + \
        list(CSRC.rglob("*.hpp")) + list(CSRC.rglob("*.cuh")) + [ROOT / "include" / "gq.h", Path(__file__)]
    return files


def _stale(target: Path, inputs) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(p.stat().st_mtime > t for p in inputs if p.exists())


def _run(cmd, verbose):
    if verbose:
        print(" ".join(str(c) for c in cmd), flush=True)
    r = subprocess.run([str(c) for c in cmd], capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"command failed: {' '.join(str(c) for c in cmd)}")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr)


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> Path:
    """Compiles libgq.so if any input is newer than it; returns its path."""
    if not force and not _stale(LIB, _all_inputs()):
        return LIB
    cuda = _cuda_home()
    nvcc = cuda / "bin" / "nvcc"
    BUILD.mkdir(parents=True, exist_ok=True)
    LIB.parent.mkdir(parents=True, exist_ok=True)
    jobs = []
    for src in HOST_SOURCES:
        obj = BUILD / (src.replace("/", "_") + ".o")
        jobs.append((["g++", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall",
                      "-Wno-unused-function", f"-I{cuda / 'include'}", "-c", CSRC / src, "-o", obj], verbose, obj))
    for src in DEVICE_SOURCES:
        obj = BUILD / (src.replace("/", "_") + ".o")
        flags = ["-O3", "-std=c++17", "--fmad=false", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler",
                 "-ffp-contract=off", *ARCH]
        if ptxas_verbose:
            flags += ["-Xptxas", "-v"]
        jobs.append(([nvcc, *flags, "-c", CSRC / src, "-o", obj], verbose or ptxas_verbose, obj))
    # the translation units are independent: compile them side by side
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 1)) as pool:
        for f in [pool.submit(_run, cmd, vb) for cmd, vb, _ in jobs]:
            f.result()
    objs = [obj for _, _, obj in jobs]
    tmp = LIB.with_suffix(".so.tmp")
    _run([nvcc, "-shared", *ARCH, "-cudart", "static", "-o", tmp, *objs, "-lpthread"], verbose)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_verbose="--ptxas" in sys.argv)
