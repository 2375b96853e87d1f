"""Multi-process replica plumbing on CPU (gloo, world size 2)."""
import os
import socket

import pytest

from sfincs_b200 import replicas


def test_partition_covers_everything_once():
    for n in (0, 1, 7, 64):
        for world in (1, 2, 3, 8):
            parts = [replicas.partition(n, world, r) for r in range(world)]
            flat = sorted(i for p in parts for i in p)
            assert flat == list(range(n))
            assert max(map(len, parts)) - min(map(len, parts)) <= 1


def test_partition_by_cost_is_balanced():
    costs = [4e4, 2.25e6, 1e6, 9e4, 5e5, 1.2e6, 3e5, 8e5]
    parts = [replicas.partition_by_cost(costs, 2, r) for r in range(2)]
    assert sorted(parts[0] + parts[1]) == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) / sum(loads) < 0.6


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = replicas.partition(7, world, rank)
        t = 1.0 + rank  # rank 1 is "slower"
        replicas.barrier()
        tmax = replicas.allreduce_max(t)
        tot = replicas.allreduce_sum(len(mine))
        out.put((rank, mine, tmax, tot))
    finally:
        dist.destroy_process_group()


def test_gloo_world2_max_over_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    assert res[0][1] + res[1][1] == list(range(7))
    assert res[0][2] == res[1][2] == 2.0
    assert res[0][3] == res[1][3] == 7.0
