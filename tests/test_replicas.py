"""Multi-rank bookkeeping of replica runs, on CPU with gloo (world size 2):
sharding covers every unit exactly once, the job time is the maximum over
ranks and unit counts are summed (the helpers bench.py uses under torchrun)."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench as replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        assert replicas.rank_world() == (rank, world)
        units = list(range(11))
        mine = replicas.shard(units)
        n_total = replicas.sum_over_ranks(len(mine))
        t_job = replicas.max_over_ranks(1.0 + rank)  # rank 1 is slower
        s = replicas.sum_over_ranks(sum(mine))
        q.put((rank, mine, n_total, t_job, s))
    finally:
        dist.destroy_process_group()


def test_replica_bookkeeping_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, m0, n0, t0, s0), (r1, m1, n1, t1, s1) = res
    assert sorted(m0 + m1) == list(range(11)) and not set(m0) & set(m1)
    assert n0 == n1 == 11
    assert t0 == t1 == 2.0
    assert s0 == s1 == sum(range(11))


def test_single_process_fallbacks():
    assert replicas.rank_world() == (0, 1)
    assert replicas.shard([1, 2, 3]) == [1, 2, 3]
    assert replicas.max_over_ranks(3.5) == 3.5
