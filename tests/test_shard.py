"""Ladders across ranks: the partition and the one collective, on two gloo
ranks over the loopback interface."""
import os
import socket

import numpy as np
import pytest


def test_partition_covers_every_ladder_once_and_balances():
    from chimera_b200.shard import ladder_cost, partition
    rng = np.random.default_rng(0)
    costs = [ladder_cost(int(rng.integers(8, 48)), 42, int(rng.choice([0, 3204])), 241, 6, 117,
                         200) for _ in range(37)]
    for world in (1, 2, 3, 8):
        parts = partition(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs) + 1e-9
        assert all(p == sorted(p) for p in parts)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, nladders, q):
    import datetime
    import torch.distributed as dist
    from chimera_b200.shard import partition, gather_summaries
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        costs = [1.0 + (i % 5) for i in range(nladders)]
        parts = partition(costs, world)
        mine = parts[rank]
        # each rank "samples" its ladders: rows (ladder id, best chi^2, rank)
        rows = np.array([[li, 100.0 - li, rank] for li in mine], float).reshape(-1, 3)
        res = gather_summaries(rows, nladders, parts)
        q.put((rank, parts, res.tolist()))
    finally:
        dist.destroy_process_group()


def test_gather_summaries_on_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port, world, nl = _free_port(), 2, 11
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, nl, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, parts, res in out:
        res = np.array(res)
        assert np.array_equal(res[:, 0], np.arange(nl))
        assert np.array_equal(res[:, 1], 100.0 - np.arange(nl))
        owner = {li: r for r, p in enumerate(parts) for li in p}
        assert all(res[li, 2] == owner[li] for li in range(nl))
        assert len(parts[0]) and len(parts[1])
