"""Host logic of the multi-GPU replicas layout, run as two gloo ranks on CPU:
the max-over-ranks timing and the round-robin query shards with the counts
gathered back in query order."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from psm_benchmark_b200.replicas import gather_counts, max_over_ranks, shard


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        times = max_over_ranks([10.0 + rank, 5.0 - rank], dist)
        items = list(range(11))
        mine = shard(items, rank, world)
        counts = [x * x for x in mine]  # stands in for per-query counts
        merged = gather_counts(counts, rank, world, dist)
        q.put((rank, times, mine, merged))
    finally:
        dist.destroy_process_group()


def test_two_ranks_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = {}
    for _ in range(world):
        rank, times, mine, merged = q.get(timeout=120)
        got[rank] = (times, mine, merged)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(world):
        assert got[r][0] == [11.0, 5.0]
    assert sorted(got[0][1] + got[1][1]) == list(range(11))
    assert got[0][2] == [x * x for x in range(11)]
    assert got[1][2] is None


def test_single_process_passthrough():
    assert max_over_ranks([1.5, 2.0]) == [1.5, 2.0]
    assert shard(range(5), 0, 1) == [0, 1, 2, 3, 4]
    assert gather_counts([3, 4], 0, 1) == [3, 4]
