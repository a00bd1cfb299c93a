"""The multi-GPU path on CPU: two gloo ranks shard the queries, each answers its shard
on its own replica of the scene (with the CPU oracle standing in for the device
kernels), and the shards put together equal the single-process answer; timings are
reduced as the maximum over ranks."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from gquery_b200.distributed import max_over_ranks, shard_bounds, shard_seed


def test_shard_bounds_partition():
    for n in (0, 1, 7, 1000, 1 << 20):
        for w in (1, 2, 3, 8):
            parts = [shard_bounds(n, r, w) for r in range(w)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
            sizes = [hi - lo for lo, hi in parts]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_bounds(10, 2, 2)
    assert shard_seed(1, 0) != shard_seed(1, 1)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, n, out_dir):
    import datetime

    import torch.distributed as dist

    import oracle
    from gquery_b200 import _lib as L
    from gquery_b200 import workloads as W
    from gquery_b200.scene import Scene
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        v, f = W.icosphere(3, amplitude=0.2, seed=4)
        scene = Scene(v, f, 3, device=None)  # each rank holds its own replica
        q = W.uniform_points(n, 3, seed=9)
        lo, hi = shard_bounds(n, rank, world)
        rec = oracle.closest_point(3, scene.ref_array(L.ARRAY_BVH_NODES), scene.ref_array(L.ARRAY_PRIMITIVES),
                                   q[lo:hi], threads=1)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), lo=lo, hi=hi, d=rec["d"], prim_id=rec["prim_id"])
        t = max_over_ranks([1.0 + rank, 5.0 - rank])
        np.save(os.path.join(out_dir, f"max{rank}.npy"), np.array(t))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce(tmp_path):
    import oracle
    from gquery_b200 import _lib as L
    from gquery_b200 import workloads as W
    from gquery_b200.scene import Scene
    n, world = 3001, 2
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, n, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    parts = [np.load(tmp_path / f"rank{r}.npz") for r in range(world)]
    assert parts[0]["lo"] == 0 and parts[0]["hi"] == parts[1]["lo"] and parts[1]["hi"] == n
    d = np.concatenate([p["d"] for p in parts])
    pid = np.concatenate([p["prim_id"] for p in parts])
    v, f = W.icosphere(3, amplitude=0.2, seed=4)
    scene = Scene(v, f, 3, device=None)
    whole = oracle.closest_point(3, scene.ref_array(L.ARRAY_BVH_NODES), scene.ref_array(L.ARRAY_PRIMITIVES),
                                 W.uniform_points(n, 3, seed=9), threads=1)
    assert np.array_equal(d.view(np.uint32), np.asarray(whole["d"], np.float32).view(np.uint32))
    assert np.array_equal(pid, whole["prim_id"])
    for r in range(world):
        assert np.load(tmp_path / f"max{r}.npy").tolist() == [2.0, 5.0]
