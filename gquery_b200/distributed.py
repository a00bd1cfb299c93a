"""One process per GPU: query sharding and timing over ranks.

Queries are independent, so the multi-GPU form of the path is data parallel with no
exchange step: every rank holds a full replica of the scene (one device-resident copy
per GPU) and answers a disjoint shard of the queries.  No collective runs in the data
path; the only collectives are the timing reduction (max over ranks) and barriers
around the timed region.  The reference has no multi-device path (DrJit runs one
device per process).
"""
from __future__ import annotations

import os
from typing import Tuple


def world() -> Tuple[int, int, int]:
    """(rank, world_size, local_rank) from the torchrun environment (1 process: 0, 1, 0)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard_bounds(n_total: int, rank: int, world_size: int) -> Tuple[int, int]:
    """Contiguous, balanced shard [lo, hi) of n_total queries for `rank`; the shards of
    all ranks partition range(n_total) and differ in size by at most one."""
    if world_size < 1 or not 0 <= rank < world_size:
        raise ValueError("rank must be in [0, world_size)")
    base, extra = divmod(int(n_total), world_size)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def shard_seed(seed: int, rank: int) -> int:
    """Seed of a rank's own synthetic query stream in weak-scaling runs (fixed work per
    rank; the streams of different ranks are disjoint)."""
    return int(seed) + 1000 * int(rank)


def max_over_ranks(values, device=None):
    """Element-wise maximum of a list of floats over all ranks (one all-reduce); the
    input itself when no process group is initialised."""
    import torch
    import torch.distributed as dist
    vals = [float(v) for v in values]
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return vals
    t = torch.tensor(vals, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]
