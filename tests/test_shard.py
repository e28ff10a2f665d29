"""Scenario sharding across GPUs (shard.py) without a GPU: the assignment is
deterministic, balanced and within the memory budget, and two gloo ranks
(world size 2, processes on CPU) each run only their share and rank 0 gathers
every scenario's result."""
import os
import socket

import pytest

import shard


def test_assign_is_deterministic_balanced_and_complete():
    costs = [5.0, 1.0, 3.0, 3.0, 8.0, 2.0, 2.0, 7.0]
    a = shard.assign(costs, 3)
    assert a == shard.assign(costs, 3)
    flat = sorted(i for r in a for i in r)
    assert flat == list(range(len(costs)))
    loads = [sum(costs[i] for i in r) for r in a]
    assert max(loads) - min(loads) <= max(costs)  # the longest-processing-time bound
    assert shard.assign(costs, 1) == [list(range(len(costs)))]


def test_assign_respects_the_memory_budget():
    costs = [10.0, 1.0, 1.0, 1.0]
    fps = [60, 30, 30, 30]
    a = shard.assign(costs, 2, fps, budget_bytes=90)
    used = [sum(fps[i] for i in r) for r in a]
    assert max(used) <= 90
    with pytest.raises(ValueError):
        shard.assign([1.0], 2, [100], budget_bytes=90)


def test_footprint_grows_with_particles():
    assert shard.footprint_bytes(2000) > shard.footprint_bytes(1000) > 0
    assert shard.footprint_bytes(1000, nodes_estimate=0) == shard.BYTES_PER_PARTICLE * 1000


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_q):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        scen = [{"Np": n, "T": t} for n, t in [(1000, 60), (50000, 30), (20000, 90), (3000, 60), (80000, 45), (500, 120)]]
        ran = []

        def run_batch(items):
            ran.extend(i for i, _ in items)
            return {i: {"rank": rank, "particle_time": s["Np"] * s["T"]} for i, s in items}

        res, shards = shard.run_sharded(scen, rank, world, cost=lambda s: s["Np"] * s["T"], run_batch=run_batch,
                                        footprint=lambda s: shard.footprint_bytes(s["Np"]), gather=shard.torch_gather())
        out_q.put((rank, sorted(ran), shards, res))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_run_their_shares_and_gather():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = {}
    for _ in range(2):
        rank, ran, shards, res = q.get(timeout=120)
        got[rank] = (ran, shards, res)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    shards = got[0][1]
    assert got[1][1] == shards  # both ranks computed the same assignment
    assert got[0][0] == shards[0] and got[1][0] == shards[1]  # each ran only its share
    assert not set(shards[0]) & set(shards[1])
    res = got[0][2]
    assert sorted(res) == list(range(6))  # rank 0 gathered every scenario
    assert all(res[i]["rank"] == (0 if i in shards[0] else 1) for i in res)
    assert got[1][2] is None
