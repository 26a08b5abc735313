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


def _step_share(oracle, specs, idx, method, substeps):
    """Steps the scenes `idx` of `specs` (small dam breaks) through the C
    oracle, a CPU stand-in for each rank's GPU, and returns {index: (x, v)}."""
    import numpy as np
    from emerald_b200 import workloads as W
    import emerald_b200 as E
    out = {}
    for k in idx:
        s = specs[k]
        sc = W.scene_for(s["nx"], s["ny"], s["seed"])
        d = sc.params.as_dict()
        cfg = E.config(sc.params)
        p = {q: d[q] for q in d if q not in ("seed", "length")}
        p.update(mass_per_particle=cfg["mass_per_particle"],
                 pressure_correction_denom=cfg["pressure_correction_denom"],
                 seconds_per_sub_step=cfg["seconds_per_sub_step"])
        sim = oracle.sim(p, sc.solid, sc.solid_volumes, sc.fluid)
        sim.begin_frame(method)
        for t in range(s.get("substeps", substeps)):
            sim.sub_step(method, np.float32(t * 2e-4), np.float32(2e-4))
        x, v = sim.state()
        out[k] = (x.tobytes(), v.tobytes())
    return out


def _small_requests(n):
    """A served stream with tiny scenes (so the oracle steps them in seconds)."""
    from emerald_b200 import workloads as W
    reqs = W.serving_requests(n, lo=64, hi=256, steps_lo=2, steps_hi=5)
    return reqs


def _serve_rank_main(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    from emerald_b200 import workloads as W
    from cpu_checkers import Oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    oracle = Oracle()
    reqs = _small_requests(12)
    mine = W.route_requests(reqs, world)[rank]
    served = _step_share(oracle, reqs, mine, "dfsph_p", 0)
    specs = [dict(s, nx=max(4, s["nx"] // 16), ny=max(4, s["ny"] // 16), substeps=2)
             for s in W.batched_specs(8)]
    sizes = [s["nx"] * s["ny"] for s in specs]
    batched = _step_share(oracle, specs, W.assign_scenes(sizes, world)[rank], "iisph", 2)
    gathered = [None] * world
    dist.all_gather_object(gathered, (mine, served, batched))
    if rank == 0:
        out.put(gathered)
    dist.barrier()
    dist.destroy_process_group()


def test_ranks_step_their_shares_as_one_process_would():
    """Two gloo ranks each take their routed share of a served request
    stream and their bin-packed share of batched scenes, and step them (the
    C oracle standing in for each rank's GPU on this CPU host). The shares
    partition the work, and every scene ends bit for bit where one process
    stepping all of them leaves it: sharding changes no result."""
    import torch.multiprocessing as mp
    from emerald_b200 import workloads as W
    from cpu_checkers import Oracle
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_serve_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    gathered = q.get(timeout=300)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    reqs = _small_requests(12)
    routed = [g[0] for g in gathered]
    assert sorted(k for lst in routed for k in lst) == list(range(len(reqs)))
    assert all(lst == sorted(lst) for lst in routed)          # arrival order kept
    oracle = Oracle()
    whole = _step_share(oracle, reqs, range(len(reqs)), "dfsph_p", 0)
    served = {k: v for g in gathered for k, v in g[1].items()}
    assert served.keys() == whole.keys()
    for k in whole:
        assert served[k] == whole[k], "request %d differs when routed" % k
    specs = [dict(s, nx=max(4, s["nx"] // 16), ny=max(4, s["ny"] // 16), substeps=2)
             for s in W.batched_specs(8)]
    whole_b = _step_share(oracle, specs, range(len(specs)), "iisph", 2)
    batched = {k: v for g in gathered for k, v in g[2].items()}
    assert batched == whole_b


def test_route_requests_balances_work():
    from emerald_b200 import workloads as W
    reqs = W.serving_requests(256)
    work = [r["nx"] * r["ny"] * r["substeps"] for r in reqs]
    for world in (1, 2, 4, 8):
        a = W.route_requests(reqs, world)
        assert a == W.route_requests(reqs, world)
        assert sorted(k for lst in a for k in lst) == list(range(len(reqs)))
        loads = [sum(work[k] for k in lst) for lst in a]
        assert max(loads) - min(loads) <= max(work)
