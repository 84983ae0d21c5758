"""Host-side multi-GPU logic on CPU: the island partition and the gather of
per-island results, with world_size 2 over gloo (no GPU: the per-rank solve
is a stub that records which islands it was given)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from pfsf_b200 import shard


def test_plan_is_balanced_complete_and_deterministic():
    rng = np.random.default_rng(0)
    sizes = (rng.lognormal(9, 1.2, 4096)).astype(np.int64)
    for world in (1, 2, 3, 8):
        plan = shard.plan_shards(sizes, world)
        flat = sorted(i for s in plan for i in s)
        assert flat == list(range(len(sizes)))
        loads = shard.shard_loads(sizes, plan)
        # LPT bound: max load <= mean + largest island
        assert max(loads) <= sum(loads) / world + sizes.max()
        assert plan == shard.plan_shards(sizes, world)
    assert shard.plan_shards([5, 5, 5], 4)[3] == []


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, sizes, out):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        def solve(indices):
            # stub of the per-rank engine call: result = (island, rank, size)
            return 10.0 + rank, {i: (i, rank, int(sizes[i])) for i in indices}

        tmax, res = shard.run_sharded(sizes, solve)
        out.put((rank, tmax, res))
    finally:
        dist.destroy_process_group()


def test_run_sharded_world_size_2():
    sizes = np.array([900, 10, 500, 470, 30, 1, 250, 249], np.int64)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, sizes, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = {}
    for _ in procs:
        rank, tmax, res = q.get(timeout=120)
        got[rank] = (tmax, res)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got[0][0] == got[1][0] == 11.0  # max over ranks
    assert got[1][1] is None
    res = got[0][1]
    plan = shard.plan_shards(sizes, 2)
    assert [r[0] for r in res] == list(range(len(sizes)))
    for i, (_, rank, size) in enumerate(res):
        assert i in plan[rank] and size == sizes[i]
