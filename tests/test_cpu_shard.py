"""Scene sharding for multi-GPU batches (bench.py --workload batch under torchrun): a static
partition by estimated cost, checked single-process and across two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from pppm_b200 import scenes


def test_partition_covers_every_scene_once_and_balances():
    specs = scenes.batch_scenes(64, 11)
    for world in (1, 2, 3, 4, 8):
        shards = scenes.shard_by_cost(specs, world)
        assert sorted(i for s in shards for i in s) == list(range(64))
        loads = [sum(scenes.scene_cost(specs[i]) for i in s) for s in shards]
        assert max(loads) <= 1.05 * sum(loads) / world
    assert scenes.shard_by_cost(specs, 4) == scenes.shard_by_cost(specs, 4)  # deterministic


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    specs = scenes.batch_scenes(64, 11)
    mine = scenes.shard_by_cost(specs, world)[rank]
    parts = [None] * world
    dist.all_gather_object(parts, [(i, specs[i]["steps"]) for i in mine])
    if rank == 0:
        out.put(parts)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_gather_every_scene():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    parts = q.get(timeout=90)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    gathered = {i: steps for part in parts for i, steps in part}
    specs = scenes.batch_scenes(64, 11)
    assert sorted(gathered) == list(range(64))
    assert all(gathered[i] == specs[i]["steps"] for i in range(64))
