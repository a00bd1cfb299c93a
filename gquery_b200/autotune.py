"""Project autotuner: picks node width, stack depth and block shape per scene and query kind.

The reference has no launch choices to make (DrJit traces one kernel per call).  Here
each scene carries a tuning table (``gq_scene_set_tuning``): per query kind the
traversal variant - binary nodes in the reference order (``exact``), binary nodes walked
once per warp of queries adjacent in the sort order (``coherent``), quantised 8-wide nodes
(``wide8``, per lane or warp-coherent) or, for silhouettes, one query per warp
(``warp``) - plus the persistent-refill budget, the threads
per block and, for the warp-coherent closest point, a 32-entry traversal stack when the
tree fits in it.  :func:`tune` times every candidate on a sample of the caller's
queries (CUDA events, median of a few launches), checks that each candidate's answers
agree with the exact traversal's (same validity, same primitive except at FP32 distance
ties), keeps the fastest in the scene's table and remembers it in a :class:`TuneCache`
keyed by the scene's shape and the sample size.  Queries with ``variant="auto"`` then
use the tuned choice.  :func:`tune_batch` does the same for the variant flags of a
:class:`~gquery_b200.batch.SceneBatch`.
"""
from __future__ import annotations

import json
import math
import os
import statistics
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Sequence

import numpy as np

KINDS = ("cp", "ray", "sil")


def candidates(kind: str, dim: int, has_wide: bool, exact_stack: int, wide_stack: int,
               has_snch: bool = True, has_wide16: bool = False) -> List[dict]:
    """Launch configurations worth timing for one query kind of one scene."""
    out: List[dict] = []
    blocks = (64, 128, 256)
    if kind == "cp":
        for b in blocks:
            out.append(dict(variant="exact", persist=0, block=b))
            out.append(dict(variant="exact", persist=1, budget=32, block=b))
            for packet in (1, 2):  # 2: the compact stack
                out.append(dict(variant="coherent", packet=packet, block=b, stack=0))
                if exact_stack <= 32:
                    out.append(dict(variant="coherent", packet=packet, block=b, stack=32))
            if has_wide:
                out.append(dict(variant="wide8", packet=0, persist=1, budget=32, block=b))
                if dim == 3:
                    for packet in (1, 2):  # 2: the compact stack
                        out.append(dict(variant="wide8", packet=packet, sorted=1, block=b))
                        out.append(dict(variant="wide8", packet=packet, sorted=0, block=b))
        if has_wide16:
            for b in blocks:
                out.append(dict(variant="wide16", persist=1, budget=32, block=b))
    elif kind == "ray":
        if has_wide16:
            for b in blocks:
                out.append(dict(variant="wide16", persist=1, budget=32, block=b))
        for b in blocks:
            out.append(dict(variant="exact", persist=1, budget=32, block=b))
            if has_wide:
                for budget in (16, 32, 64):
                    out.append(dict(variant="wide8", persist=1, budget=budget, block=b))
                out.append(dict(variant="wide8", persist=0, block=b))
        out.append(dict(variant="exact", persist=0, block=128))
        if has_wide:
            out.append(dict(variant="wide8", packet=1))  # one ray per group of 8 lanes
            for packet in (0, 2):  # per lane; 2: while-while scheduling
                out.append(dict(variant="wide8", packet=packet, sorted=0, persist=1, budget=32))  # nearest first
    elif kind == "sil":
        if not has_snch:
            return []
        for b in blocks:
            out.append(dict(variant="coherent", block=b))
            out.append(dict(variant="warp", packet=0, block=b))
            out.append(dict(variant="exact", persist=1, budget=32, block=b))
        out.append(dict(variant="exact", persist=0, block=128))
    else:
        raise ValueError(f"unknown kind {kind!r}")
    return [full_config(c) for c in out]


def full_config(c: dict) -> dict:
    d = dict(variant="exact", packet=0, sorted=1, persist=1, budget=32, block=128, stack=0)
    d.update(c)
    return d


def config_key(c: dict) -> str:
    c = full_config(c)
    return "{variant}/p{packet}s{sorted}r{persist}b{budget}t{block}k{stack}".format(**c)


class TuneCache:
    """JSON file of tuned choices keyed by scene shape, query kind and sample size."""

    def __init__(self, path: Optional[str] = None):
        self.path = path
        self.data: Dict[str, dict] = {}
        if path and os.path.exists(path):
            with open(path) as f:
                self.data = json.load(f)

    @staticmethod
    def key(info: dict, kind: str, n: int) -> str:
        bucket = 1 << max(0, int(math.log2(max(n, 1))))
        return f"d{info['dim']}/p{info['n_prims']}/n{info['n_nodes']}/w{info['n_wide_nodes']}/{kind}/q{bucket}"

    def get(self, key: str) -> Optional[dict]:
        return self.data.get(key)

    def put(self, key: str, value: dict) -> None:
        self.data[key] = value
        if self.path:
            tmp = self.path + ".tmp"
            with open(tmp, "w") as f:
                json.dump(self.data, f, indent=1, sort_keys=True)
            os.replace(tmp, self.path)


@dataclass
class TuneResult:
    kind: str
    best: dict
    table: List[dict] = field(default_factory=list)  # {"config", "ms", "agrees"} per candidate
    from_cache: bool = False


def cuda_timer(fn: Callable[[], object], steps: int = 3, warmup: int = 1) -> float:
    """Median device time in ms of `fn` (CUDA events on the current stream)."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        ts.append(a.elapsed_time(b))
    return statistics.median(ts)


def _agree(ref: dict, got: dict, rel: float = 2e-6) -> bool:
    va, vb = np.asarray(ref["valid"]).astype(bool), np.asarray(got["valid"]).astype(bool)
    if np.any(va != vb):
        return False
    both = va & vb
    da, db = np.asarray(ref["d"], np.float64)[both], np.asarray(got["d"], np.float64)[both]
    scale = np.maximum(np.maximum(np.abs(da), np.abs(db)), 1e-30)
    return bool(np.all(np.abs(da - db) <= rel * scale))


def _record_np(rec) -> dict:
    out = {}
    for k, v in vars(rec).items():
        out[k] = v.detach().cpu().numpy() if hasattr(v, "detach") else v
    return out


def _count(points, dim: int) -> int:
    """Number of points in a [D, n] or [n, D] array."""
    shape = tuple(points.shape)
    if len(shape) == 1:
        return 1
    return int(shape[0]) if shape[1] == dim else int(shape[1])


def _runner(scene, kind: str, inputs: Sequence, variant: str):
    if kind == "cp":
        return lambda: scene.closest_point(inputs[0], variant=variant)
    if kind == "ray":
        r = inputs[2] if len(inputs) > 2 else math.inf
        return lambda: scene.intersect(inputs[0], inputs[1], r, variant=variant)
    r = inputs[1] if len(inputs) > 1 else math.inf
    return lambda: scene.closest_silhouette(inputs[0], r, variant=variant)


def tune(scene, kind: str, inputs: Sequence, *, cands: Optional[List[dict]] = None,
         cache: Optional[TuneCache] = None, verify: bool = True,
         timer: Callable[[Callable[[], object]], float] = cuda_timer, apply: bool = True) -> TuneResult:
    """Times the candidates for `kind` on `inputs` (cp: (points,), ray: (origins, dirs
    [, r_max]), sil: (points [, r_max])) and stores the fastest agreeing one in the
    scene's tuning table (unless apply=False)."""
    info = scene.info
    n = _count(inputs[0], scene.dim)
    key = TuneCache.key(info, kind, n)
    if cache is not None:
        hit = cache.get(key)
        if hit is not None:
            if apply:
                scene.set_tuning(kind, **hit)
            return TuneResult(kind, hit, [], True)
    if cands is None:
        cands = candidates(kind, scene.dim, info["n_wide_nodes"] > 0, info["exact_stack"], info["wide_stack"],
                           info["n_silhouettes"] > 0, getattr(scene, "has_wide16", False))
    saved = scene.get_tuning(kind)
    ref = None
    if verify:
        scene.set_tuning(kind, **full_config(dict(variant="exact", persist=0)))
        ref = _record_np(_runner(scene, kind, inputs, "exact")())
    table = []
    try:
        for c in cands:
            scene.set_tuning(kind, **c)
            run = _runner(scene, kind, inputs, "auto")
            agrees = True
            if verify:
                agrees = _agree(ref, _record_np(run()))
            ms = timer(run) if agrees else math.inf
            table.append({"config": c, "ms": ms, "agrees": agrees})
    finally:
        scene.set_tuning(kind, **saved)
    ok = [t for t in table if t["agrees"] and math.isfinite(t["ms"])]
    if not ok:
        raise RuntimeError(f"no candidate for {kind} agreed with the exact traversal")
    best = min(ok, key=lambda t: t["ms"])["config"]
    if apply:
        scene.set_tuning(kind, **best)
    if cache is not None:
        cache.put(key, best)
    return TuneResult(kind, best, table, False)


BATCH_CHOICES = [dict(cp_variant=c, ray_variant=r, sil_variant=s)
                 for c in ("coherent", "exact", "split") for r in ("wide8", "exact")
                 for s in ("coherent", "warp", "exact")]


def tune_batch(make_batch: Callable[..., object], run_step: Callable[[object], object],
               timer: Callable[[Callable[[], object]], float] = cuda_timer,
               choices: Optional[List[dict]] = None) -> dict:
    """Times one batched step per variant choice; `make_batch(**choice)` builds a
    SceneBatch, `run_step(batch)` runs one step.  Returns {"best": choice, "table": [...]}."""
    table = []
    for ch in (choices or BATCH_CHOICES):
        b = make_batch(**ch)
        table.append({"choice": ch, "ms": timer(lambda: run_step(b))})
        del b
    best = min(table, key=lambda t: t["ms"])["choice"]
    return {"best": best, "table": table}
