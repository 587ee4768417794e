"""Instance sharding for multi-GPU batches: balanced, complete, disjoint, and the
same on every rank (checked with two gloo ranks on CPU)."""
import os

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from solidcloth_b200 import scenes
from solidcloth_b200.shard import instance_cost, partition, shard


def test_partition_balanced_and_complete():
    insts = scenes.cfg3_instances(count=512)
    costs = [instance_cost(s) for s in insts]
    for parts in (1, 2, 4, 8):
        p = partition(costs, parts)
        flat = sorted(i for q in p for i in q)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in q) for q in p]
        assert max(loads) <= 4 / 3 * (sum(costs) / parts) + max(costs)
        assert max(loads) / (sum(costs) / parts) < 1.02      # many small items: near perfect


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    insts = scenes.cfg3_instances(count=64, seed=7)
    mine = shard(insts, rank, world)
    names = [s.name for s in mine]
    gathered = [None] * world
    dist.all_gather_object(gathered, names)
    import torch
    t = torch.tensor([float(sum(s.num_vertices for s in mine))])
    dist.all_reduce(t)
    if rank == 0:
        out.put((gathered, float(t.item())))
    dist.destroy_process_group()


def test_two_gloo_ranks_cover_every_instance_once():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    gathered, total = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    insts = scenes.cfg3_instances(count=64, seed=7)
    names = [n for g in gathered for n in g]
    assert sorted(names) == sorted(s.name for s in insts)
    assert len(set(gathered[0]) & set(gathered[1])) == 0
    assert total == float(sum(s.num_vertices for s in insts))
