"""Island sharding across GPUs (one process per GPU).

Islands are independent linear systems (the reference's tick loop,
L1-native/libpfsf/src/pfsf_engine.cpp:439, carries no data between
islands), so multi-GPU is a host-side partition with no collective on the
data path: every rank plans the same partition from the island sizes,
solves its own shard through its own engine (one persistent launch), and
the per-island results (convergence, residual, failure tuples) are gathered
to rank 0 on the host.  The only collectives are small host-side gathers
and the max over ranks of the tick time.
"""
from __future__ import annotations

import heapq

import numpy as np


def plan_shards(active_voxels, world_size):
    """Longest-processing-time bin packing: islands in decreasing size go to
    the currently lightest rank (ties to the lower rank).  Returns one sorted
    list of island indices per rank.  Deterministic, so every rank computes
    the same plan without communicating."""
    sizes = np.asarray(active_voxels, np.int64)
    order = sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i))
    heap = [(0, r) for r in range(world_size)]
    shards = [[] for _ in range(world_size)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + int(sizes[i]), r))
    return [sorted(s) for s in shards]


def shard_loads(active_voxels, shards):
    sizes = np.asarray(active_voxels, np.int64)
    return [int(sizes[s].sum()) if s else 0 for s in shards]


def run_sharded(islands_active, solve_shard, group=None):
    """Runs one tick over all islands on all ranks of `group`.

    solve_shard(indices) -> (ms, {index: result}) solves this rank's islands
    (the caller's engine call) and returns its device time and per-island
    results (any picklable objects).  Returns, on rank 0, (max ms over ranks,
    results of every island in island order); on other ranks (max ms, None).
    """
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    shards = plan_shards(islands_active, world)
    ms, results = solve_shard(shards[rank])
    if set(results) != set(shards[rank]):
        raise RuntimeError("solve_shard returned results for the wrong islands")
    gathered = [None] * world if rank == 0 else None
    dist.gather_object((ms, results), gathered, dst=0, group=group)
    t = [None] * world
    dist.all_gather_object(t, ms, group=group)
    tmax = max(t)
    if rank != 0:
        return tmax, None
    merged = {}
    for _, res in gathered:
        merged.update(res)
    return tmax, [merged[i] for i in range(len(islands_active))]
