"""Instance sharding for the batched workload on several ranks (CPU, gloo,
world size 2): every rank computes the same split independently; together
the shards cover every instance exactly once and their costs balance."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from phi_b200 import configs
from phi_b200.shard import balanced_shards


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, costs, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mine = balanced_shards(costs, world)[rank]
    got = [None] * world
    dist.all_gather_object(got, mine)
    load = torch.tensor([sum(costs[i] for i in mine)], dtype=torch.float64)
    mx = load.clone()
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    tot = load.clone()
    dist.all_reduce(tot, op=dist.ReduceOp.SUM)
    if rank == 0:
        q.put((got, float(mx.item()), float(tot.item())))
    dist.destroy_process_group()


def test_shards_cover_instances_once_across_two_ranks():
    costs = [p.nodes * p.num_states ** 2 for p in configs.batched(seed=3, count=512)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    got, mx, tot = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    flat = sorted(i for part in got for i in part)
    assert flat == list(range(len(costs)))
    assert mx <= 1.01 * tot / 2


@pytest.mark.parametrize("world", [1, 3, 8])
def test_balanced_shards_properties(world):
    costs = [5, 1, 9, 3, 3, 7, 2, 8, 1, 1]
    parts = balanced_shards(costs, world)
    assert sorted(i for p in parts for i in p) == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(costs)
