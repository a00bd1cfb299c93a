#!/usr/bin/env python
"""Benchmark: 3D closest point + ray intersection on the displaced icosphere of
level 8 (1,310,720 triangles), 8,388,608 closest-point queries U[-2,2]^3 and
8,388,608 rays (origins U[-2,2]^3, directions uniform on S^2, r_max = inf).

One step = Morton-order + closest_point over all points, then Morton-order +
intersect over all rays, on the quantised 8-wide BVH.  The exact binary kernel
(gQuery's visit order) is measured beside it.  Prints one JSON line (rank 0).

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
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-compare", action="store_true", help="skip the exact and wide8 side-by-side runs")
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


def run_reference(args):
    """Reference arm: the CPU restatement of gQuery's traversal (DrJit cannot be
    installed here) on the host cores, a bounded sample per step."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from gquery_b200 import workloads as W
    V, F = W.config1_mesh()
    per_step = 16384
    q = W.uniform_points(per_step, 3, seed=1)
    o, d = W.rays(per_step, 3, seed=2)
    import oracle
    from gquery_b200 import _lib as L
    from gquery_b200.scene import Scene
    s = Scene(V, F, 3, device=None, build_snch=False, build_wide=False)
    nodes, prims = s.ref_array(L.ARRAY_BVH_NODES), s.ref_array(L.ARRAY_PRIMITIVES)
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
                       "sample": sample},
            "cpu_baseline": {"value": value, "unit": "Mqueries/s", "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "Mqueries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist
    from gquery_b200 import workloads as W
    from gquery_b200.scene import Scene

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = torch.device("cuda", local)

    def barrier():
        if world > 1:
            dist.barrier()

    n = args.n
    V, F = W.config1_mesh()
    scene = Scene(V, F, 3, device=local, build_snch=False, build_wide=True)
    # disjoint query shards per rank (weak scaling)
    q_h = W.uniform_points(n, 3, seed=1 + 1000 * rank)
    o_h, d_h = W.rays(n, 3, seed=2 + 1000 * rank)
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
        scene.order(o, out=perm_o, scratch=scratch)
        if ev:
            ev[3].record()
        scene.intersect(o, d, variant=variant, out=ray_out, order=perm_o)
        if ev:
            ev[4].record()

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
            t = torch.tensor([res["step_ms"], res["cp_ms"], res["ray_ms"]], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            res["step_ms"], res["cp_ms"], res["ray_ms"] = (float(x) for x in t.tolist())
        return res, clk

    if args.no_compare:
        plain = quant = None
    else:
        plain, _ = timed("exact", max(2, args.steps // 2), 2)
        quant, _ = timed("wide8", max(2, args.steps // 2), 2)
    main_res, clocks = timed(args.variant, args.steps, max(3, args.warmup), clocks=True)
    assert scene.device_error() == 0, "device error flag raised"

    total_q = 2 * n * world
    value = total_q / (main_res["step_ms"] / 1e3) / 1e6
    plain_value = total_q / (plain["step_ms"] / 1e3) / 1e6 if plain else None
    quant_value = total_q / (quant["step_ms"] / 1e3) / 1e6 if quant else None

    # ---- end to end through the public API with host buffers ----
    e2e = None
    if not args.no_e2e:
        qh = torch.as_tensor(q_h).pin_memory()
        oh = torch.as_tensor(o_h).pin_memory()
        dh = torch.as_tensor(d_h).pin_memory()
        host_cp = {k: torch.empty(v.shape, dtype=v.dtype).pin_memory() for k, v in vars(cp_out).items()}
        host_ray = {k: torch.empty(v.shape, dtype=v.dtype).pin_memory() for k, v in vars(ray_out).items()}
        qd, od, dd = torch.empty_like(q), torch.empty_like(o), torch.empty_like(d)
        h2d = 3 * qh.numel() * 4
        d2h = sum(t.numel() * t.element_size() for t in host_cp.values()) + \
            sum(t.numel() * t.element_size() for t in host_ray.values())

        def e2e_step():
            qd.copy_(qh, non_blocking=True)
            od.copy_(oh, non_blocking=True)
            dd.copy_(dh, non_blocking=True)
            r1 = scene.closest_point(qd, variant=args.variant, out=cp_out, scratch=scratch)
            r2 = scene.intersect(od, dd, variant=args.variant, out=ray_out, scratch=scratch)
            for k, v in vars(r1).items():
                host_cp[k].copy_(v, non_blocking=True)
            for k, v in vars(r2).items():
                host_ray[k].copy_(v, non_blocking=True)

        for _ in range(2):
            e2e_step()
        torch.cuda.synchronize()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        ks = max(2, args.steps)
        for _ in range(ks):
            e2e_step()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / ks
        if world > 1:
            t = torch.tensor([ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        e2e = {"value": total_q / (ms / 1e3) / 1e6, "unit": "Mqueries/s", "ms_per_step": ms,
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h}

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
            tr = traffic_per_query().get(f"{dominant}3d_{args.variant}")
            tuned_v = scene.get_tuning(dominant)["variant"] if args.variant == "auto" else args.variant
            roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                    "traffic": (tr * n if tr else None), "kernel": f"{dominant}3d_{tuned_v}",
                    "algorithmic_bytes_per_query": b, "peak_source": peak_kind,
                    "note": "achieved = reference binary-traversal bytes (oracle visit counts) / kernel time"}
        line = {
            "metric": METRIC, "value": value, "unit": "Mqueries/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": main_res["step_ms"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "variant": f"{args.variant}+morton", "queries_per_rank": 2 * n,
                       "parallelism": f"replicated scene, {world} query shard(s)", "l2": "flushed between steps"},
            "plain_exact": plain and {"value": plain_value, "ms_per_step": plain["step_ms"], "cp_ms": plain["cp_ms"],
                                      "ray_ms": plain["ray_ms"]},
            "quantised_wide8": quant and {"value": quant_value, "ms_per_step": quant["step_ms"],
                                          "cp_ms": quant["cp_ms"], "ray_ms": quant["ray_ms"],
                                          "vs_plain": quant_value / plain_value},
            "tuned": {"cp": scene.get_tuning("cp"), "ray": scene.get_tuning("ray"),
                      "vs_plain": value / plain_value if plain else None},
            "breakdown_ms": {k: main_res[k] for k in ("order_cp_ms", "cp_ms", "order_ray_ms", "ray_ms",
                                                      "wall_ms_per_step")},
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks,
            "gpu_launches": 4 * args.steps,
            "gpu_launches_note": "own kernels per step: 2 Morton-key + 2 traversal (CUB radix-sort kernels extra)",
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
