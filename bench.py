#!/usr/bin/env python
"""Benchmark of the geometry-query engine on one B200 (or N, weak scaling).

Headline (the JSON line's `value`): 3D closest point + ray intersection on the
displaced icosphere of level 8 (1,310,720 triangles), 8,388,608 closest-point queries
U[-2,2]^3 and 8,388,608 rays (origins U[-2,2]^3, directions uniform on S^2, r_max =
inf).  One step = point order + closest_point over all points and the rays' order (origin
and direction) + intersect over all rays, each with the scene's tuned variant, the two
kinds on two streams side by side; the same step kind after kind on one stream gives the
per-kind breakdown, and the exact binary kernel (gQuery's visit order) and the quantised
8-wide kernel are measured beside it that way.

At one GPU the same line also carries (see --sections): c0 2D closest point on the
4,096-vertex star (every GPU variant and the CPU oracle), c2 closest silhouettes on the
level-7 mesh (plain, refill, coherent), c3 512 uneven 2D scenes answered by one
batched launch per step (eager and CUDA graph) against one plain call per scene and
kind, c4 the serving runtime under open-loop Poisson load against per-request launches.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Multi-GPU (weak scaling, replicated scene, disjoint query shards, no collective in
the data path): torchrun --nproc-per-node N bench.py --gpus N
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
# hardware work queues for the serving runtime's streams (read when the CUDA context is created)
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

METRIC = "Mqueries/s (cp/ray/silhouette) quantised+batched vs plain GPU; serving p50/p99 ms"
WORKLOAD = ("closest point + ray intersection, displaced icosphere level 8 (1,310,720 triangles), "
            "8,388,608 cp queries + 8,388,608 rays per step")
# canonical record sizes (bytes) of the roofline model: reference fp32 strides x 4
S_NODE3, S_TRI = 36, 40
B_IN_CP3, B_OUT_CP3, B_IN_RAY3, B_OUT_RAY3 = 12, 41, 24, 42


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=1 << 23, help="queries of each kind per rank")
    ap.add_argument("--variant", default="auto", choices=["auto", "wide8", "coherent", "exact"])
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--ref-n", type=int, default=1 << 20,
                    help="reference arm: closest points and rays per step (a prefix of the workload)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-compare", action="store_true", help="skip the exact and wide8 side-by-side runs")
    ap.add_argument("--no-autotune", action="store_true", help="use the built-in tuning table as it is")
    ap.add_argument("--sections-only", action="store_true",
                    help="run the listed sections alone, without the headline step (for profiling them)")
    ap.add_argument("--ray-n", type=int, default=1 << 23, help="rays of the rays section")
    ap.add_argument("--sections", default="fp64,rays,c0,build,c2,c3,c4",
                    help="beside the headline (cp + rays on the level-8 mesh): fp64 FP32-vs-FP64 error on "
                         "65,536 of the headline's closest points and rays, rays: the 8-wide ray kernels (one "
                         "ray per lane or per group of 8 lanes) in origin and origin+direction order, "
                         "c0 2D closest point on the "
                         "4,096-vertex star (GPU and CPU), build host SAH vs device build of the "
                         "level-8 mesh, c2 silhouettes on the level-7 "
                         "mesh, c3 512 uneven 2D scenes in one batched launch, c4 serving 64 meshes; "
                         "comma-separated or 'none' (one GPU only)")
    ap.add_argument("--c2-n", type=int, default=1 << 22, help="silhouette queries (c2)")
    ap.add_argument("--c3-total", type=int, default=1 << 24, help="queries per batched step (c3)")
    ap.add_argument("--c4-requests", type=int, default=800, help="requests per serving trace (c4)")
    ap.add_argument("--c3-quick", action="store_true",
                    help="c3: batched launch only (no variant tuning, no per-scene comparison)")
    return ap.parse_args()


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_per_query():
    p = ROOT / "profiles" / "traffic.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except Exception:
            return {}
    return {}


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled while the timed region runs."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(V, F, q, o, d, seconds, counts=True):
    """CPU restatement of the reference traversal on all host cores, over a bounded
    prefix of the same queries; also returns the per-query visit counts."""
    import oracle
    from gquery_b200 import _lib as L
    from gquery_b200.scene import Scene
    s = Scene(V, F, 3, device=None, build_snch=False, build_wide=False)
    nodes, prims = s.ref_array(L.ARRAY_BVH_NODES), s.ref_array(L.ARRAY_PRIMITIVES)
    threads = oracle.n_threads()
    chunk = 4096
    done = 0
    t_total = 0.0
    cnt = {"cp_interior": [], "cp_tested": [], "ray_interior": [], "ray_tested": []}
    while t_total < seconds and done + chunk <= q.shape[0]:
        t0 = time.perf_counter()
        rc = oracle.closest_point(3, nodes, prims, q[done:done + chunk], counts=counts, threads=threads)
        rr = oracle.intersect(3, nodes, prims, o[done:done + chunk], d[done:done + chunk], counts=counts,
                              threads=threads)
        t_total += time.perf_counter() - t0
        done += chunk
        if counts:
            cnt["cp_interior"].append(rc["interior"])
            cnt["cp_tested"].append(rc["tested"])
            cnt["ray_interior"].append(rr["interior"])
            cnt["ray_tested"].append(rr["tested"])
    means = {k: float(np.concatenate(v).mean()) for k, v in cnt.items() if v}
    return {"value": 2 * done / t_total / 1e6, "unit": "Mqueries/s", "cores": threads,
            "kind": "port", "seconds": t_total,
            "sample": f"first {done} cp queries + first {done} rays of the same workload"}, means


def dev_ms(fn, steps, warmup, flush=None):
    """Median device time (CUDA events on the current stream) of `fn`, L2 flushed before each call."""
    import torch
    for _ in range(warmup):
        if flush is not None:
            flush.zero_()
        fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(steps):
        if flush is not None:
            flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        ts.append(a.elapsed_time(b))
    return statistics.median(ts)


def read_gbs(dev, mbytes, reps):
    """Read bandwidth of a `mbytes` MB buffer read `reps` times in one launch with L2-only
    16-byte loads (gq_read_probe): best of three, CUDA events.  A buffer that fits in L2
    (126 MB) measures L2; a larger one HBM."""
    import torch
    from gquery_b200 import _lib as L
    buf = torch.ones(mbytes << 20, dtype=torch.uint8, device=dev)
    sink = torch.zeros(1, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    run = lambda: L.check(L.lib().gq_read_probe(buf.data_ptr(), buf.numel(), reps, sink.data_ptr(), stream))  # noqa: E731
    run()
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        run()
        e1.record()
        torch.cuda.synchronize()
        best = max(best, buf.numel() * reps / (e0.elapsed_time(e1) / 1e3) / 1e9)
    return best


def fp64_error(kind, valid, d, d64):
    """FP32 answers against the FP64 brute force: validity that differs, and the error of
    the distance (closest point, silhouette: absolute; ray: relative to max(t, 1)) where
    both found one.  Silhouettes also count answers farther than the FP64 nearest by more
    than 5e-7 (the reference's cone test may skip the nearest silhouette)."""
    import torch
    v = valid.bool()
    h = torch.isfinite(d64)
    both = v & h
    diff = d.double() - d64
    err = diff.abs() / d64.clamp(min=1.0) if kind == "ray" else diff.abs()
    e = err[both]
    out = {"n": int(v.numel()), "found": int(both.sum()), "valid_differs": int((v != h).sum())}
    if e.numel():
        out.update({"max": float(e.max()), "median": float(e.median()),
                    "p99_9": float(torch.quantile(e.float(), 0.999)),
                    "unit": "relative to max(t, 1)" if kind == "ray" else "absolute"})
    if kind == "sil":
        out["farther_than_fp64"] = int((diff[both] > 5e-7).sum())
        out["nearer_than_fp64"] = int((diff[both] < -5e-7).sum())
    return out


def tie_stats(a, b, rel=2e-6):
    """Answers of a fast variant `a` against the exact traversal `b` (records of device
    tensors): validity mismatches, differing primitives split into exact ties (the same
    FP32 distance bit for bit), loose ties (distances within `rel` relative) and the rest."""
    import torch
    va, vb = a.valid.bool(), b.valid.bool()
    both = va & vb
    da, db = a.d.double(), b.d.double()
    reld = (da - db).abs() / torch.maximum(torch.maximum(da.abs(), db.abs()), torch.full_like(da, 1e-30))
    diff = both & (a.prim_id != b.prim_id)
    exact = diff & (a.d == b.d)
    return {"n": int(va.numel()), "valid_mismatch": int((va != vb).sum()), "prim_mismatch": int(diff.sum()),
            "prim_mismatch_exact_tie": int(exact.sum()),
            "prim_mismatch_loose_tie": int((diff & ~exact & (reld <= rel)).sum()),
            "prim_mismatch_not_tie": int((diff & (reld > rel)).sum()),
            "max_rel_d": float(reld[both].max()) if bool(both.any()) else 0.0}


def section_rays(args, dev, flush):
    """Rays of the headline workload over the quantised 8-wide nodes: one ray per lane and
    one ray per group of 8 lanes, each in the origins' point order (mode 0) and in the
    origin + direction order (mode 2); the records of all four must be the same."""
    import torch
    from gquery_b200 import workloads as W
    from gquery_b200.scene import Scene
    V, F = W.config1_mesh()
    s = Scene(V, F, 3, device=dev.index or 0, build_snch=False, build_wide=True)
    n = args.ray_n
    o, d = (torch.as_tensor(a).to(dev) for a in W.rays(n, 3, seed=2))
    res = {"workload": f"{n} rays U[-2,2]^3 x S^2 on the level-8 mesh, 8-wide nodes"}
    ref = None
    same = True
    for mode in (0, 2):
        order = s.ray_order(o, d, mode)
        for name, packet in (("per_lane", 0), ("group_of_8", 1)):
            s.set_tuning("ray", "wide8", packet=packet, sorted=1, persist=1)
            out = s.alloc_ray(n)
            ms = dev_ms(lambda: s.intersect(o, d, variant="wide8", out=out, order=order),
                        steps=max(1, min(args.steps, 5)), warmup=1, flush=flush)
            res[f"{name}_order{mode}"] = {"ms": ms, "mrays_per_s": n / ms / 1e3}
            rec = {k: v.clone() for k, v in vars(out).items()}
            if ref is None:
                ref = rec
            same = same and all(torch.equal(rec[k], ref[k]) for k in rec)
    res["records_identical"] = bool(same)
    assert s.device_error() == 0
    return res


def section_c0(args, dev, flush):
    """2D closest point: 4,096-vertex star polyline, 1,048,576 points U[-2,2]^2 - the
    configuration that also runs on the CPU: every GPU variant and the CPU oracle port
    on all host cores over the same points."""
    import torch
    import oracle
    from gquery_b200 import _lib as L
    from gquery_b200 import workloads as W
    from gquery_b200.scene import Scene
    V, E, Q = W.config0()
    sc = Scene(V, E, 2, device=dev.index or 0, build_snch=False)
    n = Q.shape[0]
    q = torch.as_tensor(Q).to(dev)
    order = sc.order(q)
    out = sc.alloc_cp(n)
    scratch = torch.empty(sc.scratch_bytes(n), dtype=torch.uint8, device=dev)
    res = {"workload": f"2D closest point, star polyline {E.shape[0]} segments, {n} points U[-2,2]^2"}
    for variant in ("exact", "wide8", "coherent", "auto"):
        ms = dev_ms(lambda: sc.closest_point(q, variant=variant, out=out, order=order, scratch=scratch),
                    steps=5, warmup=3, flush=flush)
        res[variant] = {"ms": ms, "mqueries_per_s": n / ms / 1e3}
    res["auto_variant"] = sc.get_tuning("cp")["variant"]
    host = Scene(V, E, 2, device=None, build_snch=False, build_wide=False)
    nodes, prims = host.ref_array(L.ARRAY_BVH_NODES), host.ref_array(L.ARRAY_PRIMITIVES)
    threads = oracle.n_threads()
    t0 = time.perf_counter()
    oracle.closest_point(2, nodes, prims, Q, threads=threads)
    cpu_s = time.perf_counter() - t0
    res["cpu_oracle"] = {"seconds": cpu_s, "mqueries_per_s": n / cpu_s / 1e6, "cores": threads, "kind": "port"}
    assert sc.device_error() == 0
    # FP32 (the exact traversal, equal to the reference's) against FP64 brute force on the
    # first 65,536 points, 65,536 rays and 65,536 silhouette points of this star
    snch = Scene(V, E, 2, device=dev.index or 0, build_snch=True)
    m = 1 << 16
    qs = q[:m]
    ro, rd = (torch.as_tensor(a).to(dev) for a in W.rays(m, 2, seed=3))
    cp = snch.closest_point(qs, variant="exact")
    ray = snch.intersect(ro, rd, variant="exact")
    sil = snch.closest_silhouette(qs, variant="exact")
    res["fp64_error"] = {
        "cp2d": fp64_error("cp", cp.valid, cp.d, snch.brute_f64("cp", qs)[0]),
        "ray2d": fp64_error("ray", ray.valid, ray.d, snch.brute_f64("ray", ro, rd)[0]),
        "sil2d": fp64_error("sil", sil.valid, sil.d, snch.brute_f64("sil", qs)[0])}
    assert snch.device_error() == 0
    return res


def section_build(args, dev, flush):
    """Scene build for the level-8 mesh: the host SAH build (the reference's builder
    algorithm) against the linear BVH built on the device, each as the binary BVH alone
    and in full (quantised 8-wide nodes and SNCH too), and closest-point / ray /
    silhouette throughput on each full scene."""
    import torch
    from gquery_b200 import workloads as W
    from gquery_b200.scene import Scene
    V, F = W.config1_mesh()
    dv = dev.index or 0
    res = {"workload": f"icosphere level 8, {F.shape[0]} triangles; 1,048,576 cp queries + rays + "
                       "silhouette points"}
    t0 = time.perf_counter()
    Scene(V, F, 3, device=dv, build_snch=False, build_wide=False)
    res["host_sah_build_s"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    host = Scene(V, F, 3, device=dv)
    res["host_full_build_s"] = time.perf_counter() - t0
    torch.cuda.synchronize()
    Scene(V, F, 3, device=dv, gpu_build=True)  # warm-up (module load, pool growth)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    Scene(V, F, 3, device=dv, gpu_build=True, build_snch=False, build_wide=False)
    torch.cuda.synchronize()
    res["device_build_s"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    devb = Scene(V, F, 3, device=dv, gpu_build=True)
    torch.cuda.synchronize()
    res["device_full_build_s"] = time.perf_counter() - t0
    res["device_tree_depth"] = devb.info["max_depth"]
    res["host_tree_depth"] = host.info["max_depth"]
    n = 1 << 20
    q = torch.as_tensor(W.uniform_points(n, 3, seed=41)).to(dev)
    o, d = (torch.as_tensor(a).to(dev) for a in W.rays(n, 3, seed=42))
    for name, sc in (("host_tree", host), ("device_tree", devb)):
        row = {}
        for variant in ("exact", "coherent"):
            ms = dev_ms(lambda: sc.closest_point(q, variant=variant), steps=3, warmup=2, flush=flush)
            row[f"cp_{variant}_mqueries_per_s"] = n / ms / 1e3
        for variant in ("exact", "wide8"):
            ms = dev_ms(lambda: sc.intersect(o, d, variant=variant), steps=3, warmup=2, flush=flush)
            row[f"ray_{variant}_mqueries_per_s"] = n / ms / 1e3
        ms = dev_ms(lambda: sc.closest_silhouette(q, variant="coherent"), steps=2, warmup=1, flush=flush)
        row["sil_coherent_mqueries_per_s"] = n / ms / 1e3
        res[name] = row
    return res


def section_c2(args, dev, flush):
    """Closest silhouette, displaced icosphere level 7 (327,680 triangles, amplitude 0.3),
    4,194,304 points U[-2,2]^3: the reference visit order one query per thread (plain),
    the same with persistent lane refill, the warp-coherent traversal and one query per
    warp."""
    import torch
    from gquery_b200 import workloads as W
    from gquery_b200.scene import Scene
    V, F = W.config2_mesh()
    t0 = time.perf_counter()
    sc = Scene(V, F, 3, device=dev.index or 0, build_snch=True, build_wide=False)
    build_s = time.perf_counter() - t0
    n = args.c2_n
    x = torch.as_tensor(W.uniform_points(n, 3, seed=31)).to(dev)
    order = sc.order(x)
    out = sc.alloc_sil(n)
    scratch = torch.empty(sc.scratch_bytes(n), dtype=torch.uint8, device=dev)
    res = {"workload": "closest silhouette, icosphere level 7 (327,680 triangles) amplitude 0.3, "
                       f"{n} points U[-2,2]^3", "build_s": build_s}
    for name, variant, persist in (("plain_exact", "exact", 0), ("exact_refill", "exact", 1),
                                   ("coherent", "coherent", 1), ("warp", "warp", 1)):
        sc.set_tuning("sil", variant, persist=persist)
        ms = dev_ms(lambda: sc.closest_silhouette(x, variant=variant, out=out, order=order, scratch=scratch),
                    steps=2 if variant == "exact" else 3, warmup=1, flush=flush)
        res[name] = {"ms": ms, "mqueries_per_s": n / ms / 1e3}
    assert sc.device_error() == 0
    # FP32 against FP64 brute force over every silhouette edge, first 65,536 points
    xs = x[:1 << 16]
    d64 = sc.brute_f64("sil", xs)[0]
    res["fp64_error"] = {}
    for variant in ("exact", "coherent"):
        r = sc.closest_silhouette(xs, variant=variant)
        res["fp64_error"][f"sil3d_{variant}"] = fp64_error("sil", r.valid, r.d, d64)
    assert sc.device_error() == 0
    res["coherent_vs_plain"] = res["plain_exact"]["ms"] / res["coherent"]["ms"]
    res["warp_vs_plain"] = res["plain_exact"]["ms"] / res["warp"]["ms"]
    return res


def section_c3(args, dev, flush):
    """512 star polylines (64 - 262,144 segments, log-uniform), 16,777,216 queries split
    50/30/20 closest point / ray / silhouette, counts proportional to segments: one
    batched launch per step (eager and CUDA-graph replay) against one plain single-scene
    call per scene and kind."""
    import torch
    from concurrent.futures import ThreadPoolExecutor
    from gquery_b200 import workloads as W
    from gquery_b200.batch import SceneBatch
    from gquery_b200.scene import Scene
    geo = W.config3_scenes()
    Q = W.config3_queries(geo, n_total=args.c3_total)
    t0 = time.perf_counter()
    with ThreadPoolExecutor(os.cpu_count() or 8) as ex:
        scenes = list(ex.map(lambda g: Scene(g[0], g[1], 2, device=dev.index or 0, build_snch=True, n_threads=1),
                             geo))
    build_s = time.perf_counter() - t0
    cp_ids, cp_pts = (torch.as_tensor(a).to(dev) for a in Q["cp"])
    ray_ids, ray_o, ray_d = (torch.as_tensor(a).to(dev) for a in Q["ray"])
    sil_ids, sil_pts = (torch.as_tensor(a).to(dev) for a in Q["sil"])
    ns = (cp_ids.numel(), ray_ids.numel(), sil_ids.numel())
    total = sum(ns)
    from gquery_b200.autotune import tune_batch
    out = None

    def make(**choice):
        return SceneBatch(scenes, max(ns), **choice)

    def step(bb):
        nonlocal out
        if out is None:
            out = bb.alloc(*ns)
        bb.run(cp=(cp_pts, cp_ids), ray=(ray_o, ray_d, ray_ids), sil=(sil_pts, sil_ids), out=out)
    t_tune = time.perf_counter()
    tb = {"best": dict(cp_variant="coherent", ray_variant="wide8", sil_variant="coherent"), "table": []} \
        if args.c3_quick else tune_batch(make, step)
    tune_s = time.perf_counter() - t_tune
    b = SceneBatch(scenes, max(ns), **tb["best"])
    if out is None:
        out = b.alloc(*ns)
    eager_ms = dev_ms(lambda: b.run(cp=(cp_pts, cp_ids), ray=(ray_o, ray_d, ray_ids), sil=(sil_pts, sil_ids),
                                    out=out), steps=5, warmup=3, flush=flush)
    kind_ms = {k: dev_ms(lambda: b.run(out=out, **a), steps=3, warmup=1, flush=flush) for k, a in
               (("cp", dict(cp=(cp_pts, cp_ids))), ("ray", dict(ray=(ray_o, ray_d, ray_ids))),
                ("sil", dict(sil=(sil_pts, sil_ids))))}
    g = b.capture(*ns)
    g.cp_points.copy_(cp_pts.t())
    g.cp_scene.copy_(cp_ids)
    g.ray_origin.copy_(ray_o.t())
    g.ray_dir.copy_(ray_d.t())
    g.ray_scene.copy_(ray_ids)
    g.sil_points.copy_(sil_pts.t())
    g.sil_scene.copy_(sil_ids)
    graph_ms = dev_ms(g.replay, steps=5, warmup=3, flush=flush)
    assert b.device_error() == 0
    # plain: one single-scene call per scene and kind (queries are grouped by scene)
    bounds = [np.searchsorted(Q[k][0], np.arange(len(scenes) + 1)) for k in ("cp", "ray", "sil")]

    def per_scene(variant):
        for i, sc in enumerate(scenes):
            a, z = bounds[0][i], bounds[0][i + 1]
            if z > a:
                sc.closest_point(cp_pts[a:z], variant=variant)
            a, z = bounds[1][i], bounds[1][i + 1]
            if z > a:
                sc.intersect(ray_o[a:z], ray_d[a:z], variant=variant)
            a, z = bounds[2][i], bounds[2][i + 1]
            if z > a:
                sc.closest_silhouette(sil_pts[a:z], variant=variant if variant == "exact" else "auto")
    if args.c3_quick:
        plain_ms = tuned_ms = None
    else:
        plain_ms = dev_ms(lambda: per_scene("exact"), steps=1, warmup=1, flush=flush)
        tuned_ms = dev_ms(lambda: per_scene("auto"), steps=1, warmup=1, flush=flush)
    mq = lambda ms: total / ms / 1e3 if ms else None  # noqa: E731
    return {"workload": f"512 star polylines, {sum(e.shape[0] for _, e in geo)} segments, {total} queries "
                        f"(cp {ns[0]}, ray {ns[1]}, sil {ns[2]})", "build_s": build_s,
            "batched_vs_tuned_per_scene": tuned_ms / graph_ms if tuned_ms else None,
            "batched_graph": {"ms": graph_ms, "mqueries_per_s": mq(graph_ms)},
            "batched_eager": {"ms": eager_ms, "mqueries_per_s": mq(eager_ms)},
            "batched_kind_alone_ms": kind_ms,
            "plain_per_scene_exact": {"ms": plain_ms, "mqueries_per_s": mq(plain_ms), "launch_calls": 3 * len(scenes)},
            "per_scene_tuned": {"ms": tuned_ms, "mqueries_per_s": mq(tuned_ms)},
            "batched_vs_plain": plain_ms / graph_ms if plain_ms else None,
            "autotune": {"best": tb["best"], "seconds": tune_s,
                         "table_ms": {"/".join(t["choice"].values()): t["ms"] for t in tb["table"]}}}


def section_c4(args, dev):
    """Serving: 64 displaced icospheres (levels 4-8) resident on the device, 120 GB
    admission budget, requests with a uniform scene, kind 50/30/20 cp/ray/silhouette and
    log-uniform 1-262,144 queries U[-2,2]^3; open-loop Poisson arrivals at fractions of
    the batched server's saturation rate; latency from scheduled arrival to results in
    the request's host arrays."""
    from concurrent.futures import ThreadPoolExecutor
    from gquery_b200 import workloads as W
    from gquery_b200.scene import Scene
    from gquery_b200.serving import HostRequest, Server, poisson_arrivals, request_mix, result_fields, summarize
    levels = W.config4_levels()
    t0 = time.perf_counter()

    def build(i):
        v, f = W.config4_scene(i, levels[i])
        return Scene(v, f, 3, device=dev.index or 0, build_snch=True, n_threads=1)
    order = sorted(range(len(levels)), key=lambda i: -levels[i])
    with ThreadPoolExecutor(os.cpu_count() or 8) as ex:
        built = dict(zip(order, ex.map(build, order)))
    scenes = [built[i] for i in range(len(levels))]
    build_s = time.perf_counter() - t0
    rng = np.random.default_rng(5)
    pool = 1 << 22
    pts = rng.uniform(-2.0, 2.0, size=(pool, 3)).astype(np.float32)
    dd = rng.standard_normal((pool, 3))
    dd = (dd / np.linalg.norm(dd, axis=1, keepdims=True)).astype(np.float32)
    pools = {k: {nm: np.zeros(pool * c, dt) for nm, (c, dt) in result_fields(k, 3).items()} for k in ("cp", "ray", "sil")}
    cursor = {"cp": 0, "ray": 0, "sil": 0}
    sc_ids, kinds, counts = request_mix(args.c4_requests, len(scenes), np.random.default_rng(1))
    reqs = []
    for s_i, k, c in zip(sc_ids, kinds, counts):
        kind = ("cp", "ray", "sil")[k]
        o = int(rng.integers(0, pool - c))
        off = cursor[kind] if cursor[kind] + c <= pool else 0
        cursor[kind] = off + c
        out = {nm: (pools[kind][nm][off * cc:(off + c) * cc].reshape(cc, c) if cc > 1 else pools[kind][nm][off:off + c])
               for nm, (cc, dt) in result_fields(kind, 3).items()}
        reqs.append(HostRequest.make(int(s_i), kind, pts[o:o + c], dd[o:o + c] if kind == "ray" else None, None,
                                     out=out))
    kind_of = np.array([r.kind for r in reqs])

    def by_kind(res):
        lat = (res["t_done"] - res["t_submit"]) * 1e3
        return {k: {"p50_ms": float(np.percentile(lat[kind_of == k], 50)),
                    "p99_ms": float(np.percentile(lat[kind_of == k], 99))} for k in ("cp", "ray", "sil")}

    level_of = np.array([levels[r.scene] for r in reqs])

    def tail(res):
        """The slowest 1% of the requests: kind, size, mesh level and where the time went
        (admission wait, wait for a step slot, step run to results in the host arrays)."""
        lat = (res["t_done"] - res["t_submit"]) * 1e3
        idx = np.argsort(-lat)[:max(1, len(lat) // 100)]
        ms = lambda a, b, i: round(float(res[b][i] - res[a][i]) * 1e3, 3)
        return [{"kind": str(kind_of[i]), "n": int(res["n"][i]), "level": int(level_of[i]),
                 "latency_ms": round(float(lat[i]), 3), "admit_ms": ms("t_submit", "t_admit", i),
                 "slot_wait_ms": ms("t_admit", "t_launch", i), "run_ms": ms("t_launch", "t_done", i)} for i in idx]

    out = {"workload": f"64 icospheres levels 4-8 ({sum(20 * 4 ** x for x in levels)} triangles), "
                       f"{len(reqs)} requests, {int(counts.sum())} queries", "build_s": build_s,
           "note": "loads are fractions of the batched server's saturation arrival rate; the plain "
                   "per-request server is run at the same arrival rate"}
    sat_rate = None
    for mode in ("batched", "per_request"):
        srv = Server(scenes, budget_bytes=120 << 30, step_queries=1 << 18, max_inflight=3,
                     per_request=(mode == "per_request"))
        srv.run_trace(reqs[:40], np.zeros(40))  # warm-up
        res = srv.run_trace(reqs, np.zeros(len(reqs)))
        sat = summarize(res)
        entry = {"saturation": {"mqueries_per_s": sat["mqueries_per_s"], "requests_per_s": sat["requests_per_s"]},
                 "loads": []}
        if sat_rate is None:
            sat_rate = sat["requests_per_s"]
        for frac in ((0.3, 0.5, 0.65, 0.8) if mode == "batched" else (0.8,)):
            r = srv.run_trace(reqs, poisson_arrivals(frac * sat_rate, len(reqs), np.random.default_rng(9)))
            sm = summarize(r)
            entry["loads"].append({"load_of_batched_peak": frac, "arrivals_per_s": frac * sat_rate,
                                   "mqueries_per_s": sm["mqueries_per_s"], "p50_ms": sm["p50_ms"],
                                   "p99_ms": sm["p99_ms"], "steps": sm["steps"], "by_kind": by_kind(r),
                                   "slowest_1pct": tail(r)})
        st = srv.stats()
        assert st["device_error"] == 0
        entry["ring_device_bytes"] = st["device_bytes"]
        out[mode] = entry
        srv.close()
    return out


def run_reference(args):
    """Reference arm: the CPU restatement of gQuery's traversal (DrJit cannot be
    installed here) on the host cores, a bounded sample per step."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from gquery_b200 import workloads as W
    V, F = W.config1_mesh()
    per_step = args.ref_n  # a prefix of the workload's queries of each kind
    q = W.uniform_points(per_step, 3, seed=1)
    o, d = W.rays(per_step, 3, seed=2)
    import oracle
    # the tree: gQuery's own builder code (oracle/_ref, compiled from its sources) when it
    # is at hand, else this project's builder, whose arrays equal it bit for bit
    # (tests/test_ref_builder.py)
    if oracle.build_ref() is not None:
        arrays = oracle.reference_build(3, V, F, snch=False)
        nodes, prims = arrays["bvh_nodes"], arrays["primitives"]
        tree = "gQuery's own builder sources (oracle/_ref/libgqref.so)"
    else:
        from gquery_b200 import _lib as L
        from gquery_b200.scene import Scene
        s = Scene(V, F, 3, device=None, build_snch=False, build_wide=False)
        nodes, prims = s.ref_array(L.ARRAY_BVH_NODES), s.ref_array(L.ARRAY_PRIMITIVES)
        tree = "this project's builder (arrays bit-identical to the reference builder's)"
    threads = oracle.n_threads()

    def step():
        oracle.closest_point(3, nodes, prims, q, threads=threads)
        oracle.intersect(3, nodes, prims, o, d, threads=threads)

    for _ in range(args.warmup):
        step()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        step()
        times.append(time.perf_counter() - t0)
    ms = 1e3 * statistics.mean(times)
    value = 2 * per_step / (ms / 1e3) / 1e6
    sample = f"{per_step} cp queries + {per_step} rays per step (prefix of the workload)"
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "Mqueries/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "engine": "CPU restatement of gQuery's traversal (oracle port)",
                       "tree": tree, "sample": sample},
            "cpu_baseline": {"value": value, "unit": "Mqueries/s", "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "Mqueries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def summary(line):
    """The headline figures (variants against plain, error, serving tail), side by side,
    at the end of the line."""
    def get(*path):
        x = line
        for k in path:
            if not isinstance(x, dict) or x.get(k) is None:
                return None
            x = x[k]
        return x
    s = {"mqps": {"plain_exact": line.get("plain_exact_mqps"), "quantised_wide8": line.get("quantised_wide8_mqps"),
                  "quantised_wide16": line.get("quantised_wide16_mqps"),
                  "tuned": line.get("value"), "e2e": get("e2e", "value"),
                  "cpu_port": get("cpu_baseline", "value")},
         "quantised_wide8_vs_plain": line.get("quantised_wide8_vs_plain"), "tuned_vs_plain": line.get("tuned_vs_plain"),
         "roofline_frac_hbm": get("roofline", "frac"), "roofline_frac_l2": get("roofline", "l2", "frac"),
         "ties_tuned_cp": {k: get("parity", "tuned", "cp", k) for k in
                           ("prim_mismatch", "prim_mismatch_exact_tie", "prim_mismatch_loose_tie",
                            "prim_mismatch_not_tie", "valid_mismatch")},
         "fp64_max_err": {k: get("fp64_error", k, "max") for k in ("cp3d_exact", "ray3d_exact")},
         "c2_coherent_mqps": get("silhouette_c2", "coherent", "mqueries_per_s"),
         "c3_batched_mqps": get("batched_c3", "batched_graph", "mqueries_per_s"),
         "c3_batched_vs_tuned_per_scene": get("batched_c3", "batched_vs_tuned_per_scene")}
    for k in ("cp2d", "ray2d", "sil2d"):
        s["fp64_max_err"][k] = get("closest_point_2d_c0", "fp64_error", k, "max")
    s["fp64_max_err"]["sil3d_exact"] = get("silhouette_c2", "fp64_error", "sil3d_exact", "max")
    loads = get("serving_c4", "batched", "loads") or []
    for ld in loads:
        if abs(ld.get("load_of_batched_peak", 0) - 0.8) < 1e-9:
            s["c4_p50_p99_ms_at_80pct"] = [ld.get("p50_ms"), ld.get("p99_ms")]
    return s


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist
    from gquery_b200 import workloads as W
    from gquery_b200.distributed import max_over_ranks, shard_seed
    from gquery_b200.distributed import world as dist_world
    from gquery_b200.scene import Scene

    rank, world, local = dist_world()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = torch.device("cuda", local)
    if args.sections_only:  # the listed sections alone (one GPU), e.g. to profile one of them
        flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
        fns = {"rays": section_rays, "c0": section_c0, "build": section_build, "c2": section_c2, "c3": section_c3}
        out = {}
        for name in [x for x in args.sections.split(",") if x and x != "none"]:
            out[name] = section_c4(args, dev) if name == "c4" else fns[name](args, dev, flush)
        print(json.dumps({"sections": out}), flush=True)
        return 0

    def barrier():
        if world > 1:
            dist.barrier()

    n = args.n
    V, F = W.config1_mesh()
    scene = Scene(V, F, 3, device=local, build_snch=False, build_wide=2)  # 8- and 16-bit child bounds
    # disjoint query shards per rank (weak scaling)
    q_h = W.uniform_points(n, 3, seed=shard_seed(1, rank))
    o_h, d_h = W.rays(n, 3, seed=shard_seed(2, rank))
    q = torch.as_tensor(q_h).to(dev)
    o = torch.as_tensor(o_h).to(dev)
    d = torch.as_tensor(d_h).to(dev)
    cp_out = scene.alloc_cp(n)
    ray_out = scene.alloc_ray(n)
    perm_q = torch.empty(n, dtype=torch.int32, device=dev)
    perm_o = torch.empty(n, dtype=torch.int32, device=dev)
    scratch = torch.empty(scene.scratch_bytes(n), dtype=torch.uint8, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2
    stream = torch.cuda.current_stream()

    def step(variant, ev=None):
        if ev:
            ev[0].record()
        scene.order(q, out=perm_q, scratch=scratch)
        if ev:
            ev[1].record()
        scene.closest_point(q, variant=variant, out=cp_out, order=perm_q)
        if ev:
            ev[2].record()
        scene.ray_order(o, d, 2, out=perm_o, scratch=scratch)
        if ev:
            ev[3].record()
        scene.intersect(o, d, variant=variant, out=ray_out, order=perm_o)
        if ev:
            ev[4].record()

    # The step's two query kinds side by side: closest points and rays on two streams that
    # fork from the step's stream after the L2 flush and join it before the step ends, the
    # rays at the lower priority.  Both traversal kernels are persistent grids sized to fill
    # the GPU, so the rays' blocks take the SMs that the closest points' blocks leave as
    # that kernel drains.
    s_cp = torch.cuda.Stream(device=dev, priority=-1)
    s_ray = torch.cuda.Stream(device=dev, priority=0)
    scratch2 = torch.empty_like(scratch)

    def step_overlapped(variant, ev=None):
        main = torch.cuda.current_stream()
        if ev:
            ev[0].record(main)
        s_cp.wait_stream(main)
        s_ray.wait_stream(main)
        scene.order(q, out=perm_q, scratch=scratch, stream=s_cp)
        scene.closest_point(q, variant=variant, out=cp_out, order=perm_q, scratch=scratch, stream=s_cp)
        scene.ray_order(o, d, 2, out=perm_o, scratch=scratch2, stream=s_ray)
        scene.intersect(o, d, variant=variant, out=ray_out, order=perm_o, scratch=scratch2, stream=s_ray)
        main.wait_stream(s_cp)
        main.wait_stream(s_ray)
        if ev:
            ev[1].record(main)

    def timed_overlapped(variant, steps, warmup, clocks=False):
        for _ in range(warmup):
            flush.zero_()
            step_overlapped(variant)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        sampler = ClockSampler(torch.cuda.current_device()) if clocks else None
        if sampler:
            sampler.start()
        evs = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(steps)]
        t_wall = time.perf_counter()
        for i in range(steps):
            flush.zero_()
            step_overlapped(variant, evs[i])
        torch.cuda.synchronize()
        t_wall = time.perf_counter() - t_wall
        barrier()
        clk = sampler.stop() if sampler else None
        res = {"step_ms": statistics.mean(e[0].elapsed_time(e[1]) for e in evs), "wall_ms_per_step": 1e3 * t_wall / steps}
        if world > 1:  # max over ranks
            res["step_ms"] = max_over_ranks([res["step_ms"]], device=dev)[0]
        return res, clk

    def timed(variant, steps, warmup, clocks=False):
        for _ in range(warmup):
            flush.zero_()
            step(variant)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        sampler = ClockSampler(torch.cuda.current_device()) if clocks else None
        if sampler:
            sampler.start()
        evs = [[torch.cuda.Event(enable_timing=True) for _ in range(5)] for _ in range(steps)]
        t_wall = time.perf_counter()
        for i in range(steps):
            flush.zero_()
            step(variant, evs[i])
        torch.cuda.synchronize()
        t_wall = time.perf_counter() - t_wall
        barrier()
        clk = sampler.stop() if sampler else None
        per = [[e[k].elapsed_time(e[k + 1]) for k in range(4)] for e in evs]
        step_ms = [sum(p) for p in per]
        res = {"step_ms": statistics.mean(step_ms), "order_cp_ms": statistics.mean(p[0] for p in per),
               "cp_ms": statistics.mean(p[1] for p in per), "order_ray_ms": statistics.mean(p[2] for p in per),
               "ray_ms": statistics.mean(p[3] for p in per), "wall_ms_per_step": 1e3 * t_wall / steps}
        if world > 1:  # max over ranks
            res["step_ms"], res["cp_ms"], res["ray_ms"] = max_over_ranks(
                [res["step_ms"], res["cp_ms"], res["ray_ms"]], device=dev)
        return res, clk

    if args.no_compare:
        plain = quant = quant16 = None
    else:
        saved = {k: scene.get_tuning(k) for k in ("cp", "ray")}
        plain, _ = timed("exact", max(2, args.steps // 2), 2)
        # each quantised form in its fastest measured configuration: 8-bit closest points
        # warp-coherent (nearest child first), 16-bit ones and all rays one lane per query
        scene.set_tuning("cp", "wide8", packet=1, sorted=0)
        scene.set_tuning("ray", "wide8", packet=0, sorted=1, persist=1)
        quant, _ = timed("wide8", max(2, args.steps // 2), 2)
        scene.set_tuning("cp", "wide16", persist=1)
        scene.set_tuning("ray", "wide16", persist=1)
        quant16, _ = timed("wide16", max(2, args.steps // 2), 2)
        for k, t in saved.items():
            scene.set_tuning(k, t["variant"], **{f: t[f] for f in ("packet", "sorted", "persist", "budget", "block",
                                                                  "stack")})
    tuning_report = None
    if args.variant == "auto" and not args.no_autotune:
        # the project's autotuner picks node width, stack depth and block shape on this
        # rank's own queries before the timed run (every candidate checked against exact)
        from gquery_b200.autotune import tune
        t_tune = time.perf_counter()
        r_cp = tune(scene, "cp", (q,), verify=True)
        r_ray = tune(scene, "ray", (o, d), verify=True)
        tuning_report = {"seconds": time.perf_counter() - t_tune,
                         "candidates": {"cp": len(r_cp.table), "ray": len(r_ray.table)},
                         "cp_table_ms": {f"{t['config']['variant']}/b{t['config']['block']}/k{t['config']['stack']}"
                                         f"/p{t['config']['packet']}s{t['config']['sorted']}r{t['config']['persist']}": t["ms"]
                                         for t in r_cp.table}}
    # the step kind after kind (per-kind times for the breakdown and the roofline), then the
    # headline: the same step with its two kinds side by side
    main_res, _ = timed(args.variant, args.steps, max(3, args.warmup))
    ovl_res, clocks = timed_overlapped(args.variant, args.steps, max(3, args.warmup), clocks=True)
    assert scene.device_error() == 0, "device error flag raised"

    # ---- parity at full size: the quantised and tuned answers against the exact ones ----
    parity = None
    if not args.no_compare:
        ex_cp, ex_ray = scene.alloc_cp(n), scene.alloc_ray(n)
        scene.closest_point(q, variant="exact", out=ex_cp)
        scene.intersect(o, d, variant="exact", out=ex_ray)
        parity = {"note": "answers on all queries of this rank against the exact traversal (gQuery's visit "
                          "order); ties: exact = the same FP32 distance, loose = within 2e-6 relative"}
        for name, variant in (("quantised_wide8", "wide8"), ("quantised_wide16", "wide16"), ("tuned", args.variant)):
            scene.closest_point(q, variant=variant, out=cp_out)
            scene.intersect(o, d, variant=variant, out=ray_out)
            parity[name] = {"cp": tie_stats(cp_out, ex_cp), "ray": tie_stats(ray_out, ex_ray)}
        del ex_cp, ex_ray
        assert scene.device_error() == 0
    fp64 = None
    sections_on = [x for x in args.sections.split(",") if x and x != "none"] if world == 1 else []
    if "fp64" in sections_on:
        m = 1 << 16
        qs, os_, ds = q[:m], o[:m], d[:m]
        d64 = scene.brute_f64("cp", qs)[0]
        t64 = scene.brute_f64("ray", os_, ds)[0]
        fp64 = {"workload": f"first {m} closest points and rays of the headline workload, FP64 brute force over "
                            "all 1,310,720 triangles"}
        for variant in ("exact", args.variant):
            rc = scene.closest_point(qs, variant=variant)
            rr = scene.intersect(os_, ds, variant=variant)
            fp64[f"cp3d_{variant}"] = fp64_error("cp", rc.valid, rc.d, d64)
            fp64[f"ray3d_{variant}"] = fp64_error("ray", rr.valid, rr.d, t64)
        assert scene.device_error() == 0

    total_q = 2 * n * world
    value = total_q / (ovl_res["step_ms"] / 1e3) / 1e6
    serial_value = total_q / (main_res["step_ms"] / 1e3) / 1e6
    plain_value = total_q / (plain["step_ms"] / 1e3) / 1e6 if plain else None
    quant_value = total_q / (quant["step_ms"] / 1e3) / 1e6 if quant else None
    quant16_value = total_q / (quant16["step_ms"] / 1e3) / 1e6 if quant16 else None

    # ---- end to end through the public API with host buffers ----
    # Every step copies its inputs from pinned host memory, answers them and copies every
    # record field back to pinned host memory.  Steps alternate between two lanes (own
    # device buffers, own streams), so one step's copies overlap another's traversals;
    # within a step the ray inputs go up while closest points run and the closest-point
    # records come back while rays run.
    e2e = None
    if not args.no_e2e:
        qh = torch.as_tensor(q_h).pin_memory()
        oh = torch.as_tensor(o_h).pin_memory()
        dh = torch.as_tensor(d_h).pin_memory()

        class Lane:
            def __init__(self, first):
                self.qd, self.od, self.dd = torch.empty_like(q), torch.empty_like(o), torch.empty_like(d)
                self.cp = cp_out if first else scene.alloc_cp(n)
                self.ray = ray_out if first else scene.alloc_ray(n)
                self.scratch = scratch if first else torch.empty_like(scratch)
                self.perm_q = torch.empty(n, dtype=torch.int32, device=dev)
                self.perm_o = torch.empty(n, dtype=torch.int32, device=dev)
                self.host_cp = {k: torch.empty(v.shape, dtype=v.dtype).pin_memory() for k, v in vars(self.cp).items()}
                self.host_ray = {k: torch.empty(v.shape, dtype=v.dtype).pin_memory() for k, v in vars(self.ray).items()}
                self.s_in, self.s_run, self.s_out = (torch.cuda.Stream(device=dev) for _ in range(3))
                self.ev = {k: torch.cuda.Event() for k in ("q", "od", "cp", "ray", "done")}
                self.used = False

        lanes = [Lane(True), Lane(False)]
        h2d = 3 * qh.numel() * 4
        d2h = sum(t.numel() * t.element_size() for t in lanes[0].host_cp.values()) + \
            sum(t.numel() * t.element_size() for t in lanes[0].host_ray.values())

        def e2e_step(ln, start_ev):
            ev = ln.ev
            with torch.cuda.stream(ln.s_in):
                ln.s_in.wait_event(start_ev)
                if ln.used:
                    ln.s_in.wait_event(ev["ray"])  # previous step of this lane has read its inputs
                ln.qd.copy_(qh, non_blocking=True)
                ev["q"].record(ln.s_in)
                ln.od.copy_(oh, non_blocking=True)
                ln.dd.copy_(dh, non_blocking=True)
                ev["od"].record(ln.s_in)
            r = ln.s_run
            r.wait_event(ev["q"])
            if ln.used:
                r.wait_event(ev["done"])  # previous records of this lane are back on the host
            with torch.cuda.stream(r):
                flush.zero_()  # L2 flushed before every step, as in the device-timed run
            scene.order(ln.qd, out=ln.perm_q, scratch=ln.scratch, stream=r)
            scene.closest_point(ln.qd, variant=args.variant, out=ln.cp, order=ln.perm_q, scratch=ln.scratch, stream=r)
            ev["cp"].record(r)
            r.wait_event(ev["od"])
            scene.ray_order(ln.od, ln.dd, 2, out=ln.perm_o, scratch=ln.scratch, stream=r)
            scene.intersect(ln.od, ln.dd, variant=args.variant, out=ln.ray, order=ln.perm_o, scratch=ln.scratch,
                            stream=r)
            ev["ray"].record(r)
            with torch.cuda.stream(ln.s_out):
                ln.s_out.wait_event(ev["cp"])
                for k, v in vars(ln.cp).items():
                    ln.host_cp[k].copy_(v, non_blocking=True)
                ln.s_out.wait_event(ev["ray"])
                for k, v in vars(ln.ray).items():
                    ln.host_ray[k].copy_(v, non_blocking=True)
                ev["done"].record(ln.s_out)
            ln.used = True

        def e2e_run(k):
            cur = torch.cuda.current_stream()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(cur)
            for i in range(k):
                e2e_step(lanes[i % 2], e0)
            for ln in lanes:
                if ln.used:
                    cur.wait_event(ln.ev["done"])
            e1.record(cur)
            torch.cuda.synchronize()
            return e0.elapsed_time(e1)

        e2e_run(4)  # warm-up
        barrier()
        ks = max(4, args.steps)
        ms = e2e_run(ks) / ks
        if world > 1:
            ms = max_over_ranks([ms], device=dev)[0]
        # the records that came back equal the device records of the timed run
        ok = all(torch.equal(lanes[0].host_cp[k], v.cpu()) for k, v in vars(lanes[0].cp).items())
        e2e = {"value": total_q / (ms / 1e3) / 1e6, "unit": "Mqueries/s", "ms_per_step": ms,
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "lanes": 2, "host_records_match": ok,
               "l2": "flushed before every step (a 256 MB write on the step's stream, inside the timed region)",
               "note": "public API (Scene.order / closest_point / intersect) on pinned host buffers; steps "
                       "alternate between two lanes so copies overlap traversals"}

    line = None
    if rank == 0:
        cpu, means = (None, {})
        if world == 1 and not args.no_cpu_baseline:
            cpu, means = cpu_baseline(V, F, q_h, o_h, d_h, args.cpu_seconds)
        peak, peak_kind = measured_peaks()
        roof = None
        if means:
            b_cp = B_IN_CP3 + B_OUT_CP3 + S_NODE3 * (1 + 2 * means["cp_interior"]) + S_TRI * means["cp_tested"]
            b_ray = B_IN_RAY3 + B_OUT_RAY3 + S_NODE3 * (1 + 2 * means["ray_interior"]) + S_TRI * means["ray_tested"]
            dominant = "cp" if main_res["cp_ms"] >= main_res["ray_ms"] else "ray"
            b = b_cp if dominant == "cp" else b_ray
            t_ms = main_res[f"{dominant}_ms"]
            achieved = b * n / (t_ms / 1e3) / 1e9
            tuned_v = scene.get_tuning(dominant)["variant"] if args.variant == "auto" else args.variant
            tr = traffic_per_query().get(f"{dominant}3d_{tuned_v}")
            l2_peak = read_gbs(dev, 48, 64)
            prof = traffic_per_query().get(f"{dominant}3d_{tuned_v}_counters", {})
            roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                    "traffic": (tr * n if tr else None), "kernel": f"{dominant}3d_{tuned_v}",
                    "traffic_note": "DRAM bytes per query from an ncu capture at 1,048,576 queries "
                                    "(profiles/traffic.json), scaled to the launch's query count",
                    "algorithmic_bytes_per_query": b, "peak_source": peak_kind,
                    "note": "achieved = reference binary-traversal bytes (oracle visit counts) / kernel time; "
                            "those bytes are served from L2 and L1, so the level that serves them is below",
                    "l2": {"peak": l2_peak, "peak_source": "measured in this run: L2-only reads of a 48 MB "
                                                            "buffer, 64 passes in one launch (gq_read_probe)",
                           "frac": achieved / l2_peak},
                    "dram": {"achieved": (tr * n / (t_ms / 1e3) / 1e9) if tr else None,
                             "frac": (tr * n / (t_ms / 1e3) / 1e9 / peak) if tr else None},
                    "binding": prof or None}
        line = {
            "metric": METRIC, "value": value, "unit": "Mqueries/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": ovl_res["step_ms"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "variant": f"{args.variant}+morton", "queries_per_rank": 2 * n,
                       "parallelism": f"replicated scene, {world} query shard(s)", "l2": "flushed between steps",
                       "streams": "a step's closest points and rays on two streams, the rays at lower priority"},
            "plain_exact": plain and {"value": plain_value, "ms_per_step": plain["step_ms"], "cp_ms": plain["cp_ms"],
                                      "ray_ms": plain["ray_ms"]},
            "quantised_wide8": quant and {"value": quant_value, "ms_per_step": quant["step_ms"],
                                          "cp_ms": quant["cp_ms"], "ray_ms": quant["ray_ms"],
                                          "vs_plain": quant_value / plain_value},
            "quantised_wide16": quant16 and {"value": quant16_value, "ms_per_step": quant16["step_ms"],
                                             "cp_ms": quant16["cp_ms"], "ray_ms": quant16["ray_ms"],
                                             "vs_plain": quant16_value / plain_value},
            "tuned": {"cp": scene.get_tuning("cp"), "ray": scene.get_tuning("ray"),
                      "vs_plain": serial_value / plain_value if plain else None, "autotune": tuning_report,
                      "vs_plain_note": "kind after kind, as the plain line runs",
                      "kind_after_kind": {"value": serial_value, "ms_per_step": main_res["step_ms"]},
                      "overlap_gain": main_res["step_ms"] / ovl_res["step_ms"],
                      "wall_ms_per_step": ovl_res["wall_ms_per_step"]},
            "breakdown_ms": {k: main_res[k] for k in ("order_cp_ms", "cp_ms", "order_ray_ms", "ray_ms",
                                                      "wall_ms_per_step")},
            "breakdown_note": "the step kind after kind on one stream, as the plain and quantised lines run",
            "plain_exact_mqps": plain_value, "quantised_wide8_mqps": quant_value,
            "quantised_wide16_mqps": quant16_value,
            "quantised_wide8_vs_plain": quant_value / plain_value if plain else None,
            "quantised_wide16_vs_plain": quant16_value / plain_value if plain else None,
            "tuned_vs_plain": serial_value / plain_value if plain else None,
            "parity": parity, "fp64_error": fp64,
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks,
            "gpu_launches": 4 * args.steps,
            "gpu_launches_note": "own kernels per step: 1 point-key + 1 ray-key + 2 traversal (CUB radix-sort kernels extra)",
        }
        sections = sections_on
        flush_buf = flush
        for name, fn in (("rays", lambda: section_rays(args, dev, flush_buf)),
                         ("c0", lambda: section_c0(args, dev, flush_buf)),
                         ("build", lambda: section_build(args, dev, flush_buf)),
                         ("c2", lambda: section_c2(args, dev, flush_buf)), ("c3", lambda: section_c3(args, dev, flush_buf)),
                         ("c4", lambda: section_c4(args, dev))):
            if name in sections:
                key = {"rays": "rays_8wide", "c0": "closest_point_2d_c0", "build": "scene_build",
                       "c2": "silhouette_c2", "c3": "batched_c3", "c4": "serving_c4"}[name]
                t_sec = time.perf_counter()
                line[key] = fn()
                line[key]["section_wall_s"] = time.perf_counter() - t_sec
        line["summary"] = summary(line)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
