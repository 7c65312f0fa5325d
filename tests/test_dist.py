"""Replicas path on CPU: two gloo ranks shard independent work units and reduce
timings (max) and counts (sum), as bench.py does over NCCL with one GPU per rank."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from h2pack_b200 import dist as hd


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def worker(rank, world_size, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world_size),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world_size)
    try:
        items = list(range(11))
        mine = hd.shard(items, rank, world_size)
        t = hd.max_over_ranks(1.5 + rank)              # slowest rank sets the time
        n = hd.sum_over_ranks(len(mine))               # every unit counted once
        out.put((rank, mine, t, n, hd.world()))
    finally:
        dist.destroy_process_group()


def test_two_rank_sharding_and_reductions():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    ps = [ctx.Process(target=worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, m0, t0, n0, w0), (r1, m1, t1, n1, w1) = res
    assert sorted(m0 + m1) == list(range(11)) and not set(m0) & set(m1)
    assert t0 == t1 == 2.5 and n0 == n1 == 11
    assert w0 == (2, 0, 0) and w1 == (2, 1, 1)


def test_shard_by_cost_balances():
    parts = hd.shard_by_cost([10, 1, 1, 1, 9, 2], 2)
    loads = sorted(sum([10, 1, 1, 1, 9, 2][i] for i in p) for p in parts)
    assert loads == [12, 12] and sorted(i for p in parts for i in p) == list(range(6))
