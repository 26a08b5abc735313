"""Scene sharding across ranks for the batched workload (2 gloo ranks on
CPU): every scene goes to exactly one rank, loads balance, and the timing
reduction is the max over ranks, as bench.py does on NCCL."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    import torch
    import torch.distributed as dist
    from emerald_b200 import workloads as W
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    specs = W.batched_specs(64 * world)
    sizes = [s["nx"] * s["ny"] for s in specs]
    mine = W.assign_scenes(sizes, world)[rank]
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    t = torch.tensor([float(100 + rank)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    if rank == 0:
        out.put((gathered, sizes, float(t.item())))
    dist.barrier()
    dist.destroy_process_group()


def test_scene_shards_over_two_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    gathered, sizes, tmax = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    flat = sorted(k for lst in gathered for k in lst)
    assert flat == list(range(len(sizes)))          # a partition of the scenes
    loads = [sum(sizes[k] for k in lst) for lst in gathered]
    assert max(loads) - min(loads) <= max(sizes)     # greedy bound
    assert tmax == 101.0


def test_assign_scenes_is_deterministic_and_balanced():
    from emerald_b200 import workloads as W
    sizes = [s["nx"] * s["ny"] for s in W.batched_specs(512)]
    for world in (1, 2, 4, 8):
        a = W.assign_scenes(sizes, world)
        assert a == W.assign_scenes(sizes, world)
        loads = [sum(sizes[k] for k in lst) for lst in a]
        assert sorted(k for lst in a for k in lst) == list(range(512))
        assert max(loads) <= sum(sizes) / world + max(sizes)
