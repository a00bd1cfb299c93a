"""Serving: requests of any size against device-resident scenes, continuously batched.

The reference has no serving layer: each Polyline / Mesh call answers one batch of
queries on one scene (mesh.py:87, 120, 138).  :class:`Server` wraps the native runtime
of libgq.so (``gq_server_*``): a worker thread admits requests into per-kind device
rings by memory budget, copies their queries up while earlier steps compute, answers
everything admitted in one batched launch per step (all scenes, all query kinds), and
returns results to the requests' host arrays.  ``per_request=True`` gives the plain
form for comparison: one single-scene launch per request through the same pipeline.

The load helpers (:func:`poisson_arrivals`, :func:`request_mix`, :func:`summarize`)
are plain numpy so the open-loop experiment can be planned and checked on the host.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import _lib as L
from .scene import Scene

KIND_IDS = {"cp": L.KIND_CLOSEST_POINT, "ray": L.KIND_INTERSECT, "sil": L.KIND_SILHOUETTE}
KIND_NAMES = {v: k for k, v in KIND_IDS.items()}


def result_fields(kind: str, dim: int) -> Dict[str, tuple]:
    """Host result arrays of one request: name -> (components, dtype); names follow the
    reference's records (ClosestPointRecord[3D], Intersection[3D],
    ClosestSilhouettePointRecord[3D])."""
    t = "t" if dim == 2 else "uv"
    if kind == "cp":
        return {"valid": (1, np.bool_), "p": (dim, np.float32), "n": (dim, np.float32), t: (dim - 1, np.float32),
                "d": (1, np.float32), "prim_id": (1, np.int32)}
    if kind == "ray":
        return {"valid": (1, np.bool_), "p": (dim, np.float32), "n": (dim, np.float32), t: (dim - 1, np.float32),
                "d": (1, np.float32), "prim_id": (1, np.int32), "on_boundary": (1, np.bool_)}
    return {"valid": (1, np.bool_), "p": (dim, np.float32), "d": (1, np.float32), "prim_id": (1, np.int32)}


@dataclass
class HostRequest:
    """One request: scene index, kind, host inputs ([n, D] float32) and host result
    arrays (filled when the request completes)."""
    scene: int
    kind: str
    a: np.ndarray
    b: Optional[np.ndarray] = None
    r_max: Optional[np.ndarray] = None
    out: Dict[str, np.ndarray] = field(default_factory=dict)
    completion: Optional[dict] = None

    @property
    def n(self) -> int:
        return int(self.a.shape[0])

    @staticmethod
    def make(scene: int, kind: str, a, b=None, r_max=None, dim: int = 3, out: Optional[dict] = None):
        """`out` may supply the result arrays (contiguous, shapes of result_fields)."""
        a = np.ascontiguousarray(a, np.float32).reshape(-1, dim)
        b = None if b is None else np.ascontiguousarray(b, np.float32).reshape(-1, dim)
        r = None if r_max is None else np.ascontiguousarray(r_max, np.float32).reshape(-1)
        n = a.shape[0]
        if out is None:
            out = {}
            for name, (c, dt) in result_fields(kind, dim).items():
                out[name] = np.zeros((c, n) if c > 1 else (n,), dt)
        return HostRequest(scene, kind, a, b, r, out)

    def struct(self) -> L.Request:
        o = self.out

        def ptr(name):
            x = o.get(name)
            return None if x is None else x.ctypes.data

        t = ptr("t") if "t" in o else ptr("uv")
        cp = L.CpOut(ptr("valid"), ptr("p"), ptr("n"), t, ptr("d"), ptr("prim_id")) if self.kind == "cp" else L.CpOut()
        ray = (L.RayOut(ptr("valid"), ptr("p"), ptr("n"), t, ptr("d"), ptr("prim_id"), ptr("on_boundary"))
               if self.kind == "ray" else L.RayOut())
        sil = L.SilOut(ptr("valid"), ptr("p"), ptr("d"), ptr("prim_id")) if self.kind == "sil" else L.SilOut()
        return L.Request(self.scene, KIND_IDS[self.kind], self.n, self.a.ctypes.data,
                         None if self.b is None else self.b.ctypes.data,
                         None if self.r_max is None else self.r_max.ctypes.data, cp, ray, sil, 0)


def _completion_dict(c: L.Completion) -> dict:
    return {"t_submit": c.t_submit, "t_admit": c.t_admit, "t_launch": c.t_launch, "t_done": c.t_done,
            "latency": c.t_done - c.t_submit, "n": c.n, "kind": KIND_NAMES.get(c.kind), "step": c.step,
            "status": c.status}


class Server:
    """Continuous-batching server over ``scenes`` (same dimension and device).

    budget_bytes: device bytes the request rings may hold (the admission budget);
    ring_queries: ring capacity per kind (cp, ray, sil); step_queries: most queries of
    one kind per step and the largest request; max_inflight: closest-point / ray step
    slots (streams); silhouette steps have sil_slots slots of their own on the lowest
    stream priority, sil_step_queries queries per step; in the default "warp" form each
    query is a block that exits when answered, so closest-point / ray blocks are placed
    first and silhouettes fill the rest of the GPU, while the persistent forms hold at
    most sil_share of the GPU together (above 1 they may oversubscribe it; each slot at
    most all of it).  Served requests are sparse (few
    queries per scene per step), so closest points default to one lane per query in the
    reference order with long traversals taken over one per warp ("split": cheaper than
    a warp-coherent walk when neighbours are far apart, and the slowest query no longer
    sets the step time) and silhouettes to one query per warp ("warp": bounds the
    latency of far-reaching ones).

    large_queries: requests of at least this many queries form a second size class
    (half of each kind's ring, large_slots slots per kind group, lower stream
    priorities), so small requests never share a step with large ones and their blocks
    are placed first; a negative value keeps one class.  large_share caps the
    persistent grid of a large closest-point / ray step; copy_threads: host threads
    for staging queries and scattering results (0: about half the cores, at most 8)."""

    def __init__(self, scenes: Sequence[Scene], *, budget_bytes: int = 0, ring_queries=(1 << 22,) * 3,
                 step_queries: int = 1 << 19, max_inflight: int = 3, per_request: bool = False,
                 cp_variant: str = "split", ray_variant: str = "wide8", sil_variant: str = "warp",
                 sil_share: float = 1.5, sil_slots: int = 3, sil_step_queries: int = 1 << 15,
                 large_queries: int = 1 << 15, large_slots: int = 2, large_share: float = 1.0,
                 copy_threads: int = 0):
        self.scenes = list(scenes)
        self.dim = self.scenes[0].dim
        flags = (L.SERVER_PER_REQUEST if per_request else 0) | \
            (L.BATCH_CP_EXACT if cp_variant == "exact" else L.BATCH_CP_SPLIT if cp_variant == "split" else 0) | \
            (L.BATCH_RAY_EXACT if ray_variant == "exact" else 0) | \
            (L.BATCH_SIL_EXACT if sil_variant == "exact" else L.BATCH_SIL_WARP if sil_variant == "warp" else
             L.BATCH_SIL_SPLIT if sil_variant == "split" else 0)
        rq = [int(ring_queries)] * 3 if isinstance(ring_queries, int) else [int(x) for x in ring_queries]
        opts = L.ServerOpts(int(budget_bytes), (C.c_int64 * 3)(*rq), int(step_queries), int(max_inflight), flags,
                            float(sil_share), int(sil_slots), int(sil_step_queries), int(large_queries),
                            int(large_slots), float(large_share), int(copy_threads))
        arr = (C.c_void_p * len(self.scenes))(*[s.handle.value for s in self.scenes])
        h = C.c_void_p()
        L.check(L.lib().gq_server_create(arr, len(self.scenes), C.byref(opts), C.byref(h)))
        self._h = h
        self._live: Dict[int, HostRequest] = {}
        self._next_tag = 1

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            L.lib().gq_server_free(self._h)
            self._h = None
            self._live.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, req: HostRequest) -> int:
        s = req.struct()
        tag = self._next_tag
        self._next_tag += 1
        s.tag = tag
        self._live[tag] = req
        try:
            L.check(L.lib().gq_server_submit(self._h, C.byref(s)))
        except Exception:
            del self._live[tag]
            raise
        return tag

    def poll(self) -> List[HostRequest]:
        buf = (L.Completion * 256)()
        done = []
        while True:
            cnt = C.c_int64()
            L.check(L.lib().gq_server_poll(self._h, buf, 256, C.byref(cnt)))
            for i in range(cnt.value):
                req = self._live.pop(int(buf[i].tag))
                req.completion = _completion_dict(buf[i])
                done.append(req)
            if cnt.value < 256:
                return done

    def wait_idle(self, timeout: float = 120.0) -> List[HostRequest]:
        L.check(L.lib().gq_server_wait_idle(self._h, float(timeout)))
        return self.poll()

    def stats(self) -> dict:
        st = L.ServerStats()
        L.check(L.lib().gq_server_get_stats(self._h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in L.ServerStats._fields_}

    def run_trace(self, reqs: Sequence[HostRequest], t_arrival, timeout: float = 600.0) -> dict:
        """Open loop on an otherwise idle server: request i is submitted t_arrival[i]
        seconds after the start by the native driver.  Returns per-request arrays."""
        n = len(reqs)
        arr = (L.Request * n)(*[r.struct() for r in reqs])
        t = np.ascontiguousarray(t_arrival, np.float64)
        out = (L.Completion * n)()
        L.check(L.lib().gq_server_run_trace(self._h, arr, t.ctypes.data, n, out, float(timeout)))
        res = {k: np.array([getattr(out[i], k) for i in range(n)])
               for k in ("t_submit", "t_admit", "t_launch", "t_done", "n", "kind", "step", "status")}
        for i, r in enumerate(reqs):
            r.completion = _completion_dict(out[i])
        return res


# ---------------------------------------------------------------- load helpers

def poisson_arrivals(rate: float, n: int, rng: np.random.Generator) -> np.ndarray:
    """Arrival times (seconds from 0) of an open-loop Poisson process of `rate` per second."""
    if not math.isfinite(rate):
        return np.zeros(n)
    return np.cumsum(rng.exponential(1.0 / rate, size=n))


def request_mix(n_req: int, n_scenes: int, rng: np.random.Generator, max_queries: int = 262144,
                mix=(0.5, 0.3, 0.2)):
    """Scene (uniform), kind (cp/ray/sil by `mix`) and query count (log-uniform in
    [1, max_queries]) of each request."""
    scenes = rng.integers(0, n_scenes, size=n_req)
    kinds = rng.choice(3, size=n_req, p=np.asarray(mix) / np.sum(mix))
    counts = np.floor(np.exp(rng.uniform(0.0, math.log(max_queries + 1), size=n_req))).astype(np.int64)
    counts = np.clip(counts, 1, max_queries)
    return scenes.astype(np.int32), kinds.astype(np.int32), counts


def summarize(res: dict) -> dict:
    """Latency percentiles (ms) and throughput (Mqueries/s from the first arrival to the
    last completion)."""
    lat = (res["t_done"] - res["t_submit"]) * 1e3
    span = float(res["t_done"].max() - res["t_submit"].min())
    q = float(res["n"].sum())
    return {"requests": int(lat.size), "queries": int(q), "p50_ms": float(np.percentile(lat, 50)),
            "p90_ms": float(np.percentile(lat, 90)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "max_ms": float(lat.max()),
            "mqueries_per_s": q / span / 1e6 if span > 0 else float("inf"),
            "requests_per_s": lat.size / span if span > 0 else float("inf"),
            "steps": int(np.unique(res["step"]).size)}


# ---------------------------------------------------------------- several GPUs

def place_scenes(scene_bytes: Sequence[int], budgets: Sequence[int]) -> List[int]:
    """Scene affinity for serving on several GPUs: device index of every scene, chosen so
    that each device's scenes fit its budget (largest scene first, onto the device with
    the most room left; ties to the lower index).  Raises ValueError when a scene fits
    on no device."""
    room = [int(b) for b in budgets]
    if not room:
        raise ValueError("no devices")
    place = [-1] * len(scene_bytes)
    for i in sorted(range(len(scene_bytes)), key=lambda k: (-int(scene_bytes[k]), k)):
        d = max(range(len(room)), key=lambda k: (room[k], -k))
        if room[d] < int(scene_bytes[i]):
            raise ValueError(f"scene {i} ({int(scene_bytes[i])} bytes) fits on no device")
        room[d] -= int(scene_bytes[i])
        place[i] = d
    return place


class Router:
    """Requests to the GPU that holds their scene: one :class:`Server` per device over that
    device's scenes (each scene built or loaded on its device, e.g. placed by
    :func:`place_scenes`).  `scenes_by_device[d]` lists the global scene indices on
    device d; requests name global scene indices."""

    def __init__(self, scenes: Sequence[Scene], **server_kw):
        by_dev: Dict[int, List[int]] = {}
        for i, s in enumerate(scenes):
            by_dev.setdefault(int(s.device), []).append(i)
        self.route: Dict[int, tuple] = {}
        self.servers: Dict[int, Server] = {}
        for d, idx in sorted(by_dev.items()):
            self.servers[d] = Server([scenes[i] for i in idx], **server_kw)
            for local, g in enumerate(idx):
                self.route[g] = (d, local)

    def submit(self, req: HostRequest) -> tuple:
        if req.scene not in self.route:
            raise ValueError(f"scene index {req.scene} is not served")
        d, local = self.route[req.scene]
        global_scene = req.scene
        req.scene = local
        try:
            return d, self.servers[d].submit(req)
        finally:
            req.scene = global_scene

    def wait_idle(self, timeout: float = 120.0) -> List[HostRequest]:
        done: List[HostRequest] = []
        for srv in self.servers.values():
            done += srv.wait_idle(timeout)
        return done

    def close(self):
        for srv in self.servers.values():
            srv.close()
