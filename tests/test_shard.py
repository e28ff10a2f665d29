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


def test_release_estimate_tracks_the_sampled_count():
    """Sharding a releases-only ensemble balances on the particle count an
    ELLIPSE / RECTANGLE release will give (4 per covered cell); it must track
    the count the reference's UNIFORM setup produces."""
    import workloads as W
    z = W.fractal_slope_dem(512, 2.0, seed=5, rms=3.0, x_plane_end=600.0, ease_m=200.0)
    rels = [
        {"type": "ELLIPSE", "center": (300.0, 500.0), "rx": 80.0, "ry": 40.0, "rotation_deg": 30.0, "h0": 2.0},
        {"type": "ELLIPSE", "center": (250.0, 300.0), "rx": 25.0, "ry": 60.0, "rotation_deg": 0.0, "h0": 1.0},
        {"type": "RECTANGLE", "center": (200.0, 700.0), "Lx": 60.0, "Ly": 30.0, "rotation_deg": 10.0, "h0": 1.5},
    ]
    for rel in rels:
        n = len(W.release_particles(z, 2.0, rel, 300.0)["h"])
        est = W.release_particle_estimate(rel, 2.0)
        assert abs(est - n) <= 0.05 * n, (rel["type"], est, n)


def test_config4_releases_match_its_particle_scenarios():
    """config4(particles=False) draws the same scenarios as config4(): the
    same configurations, and releases whose estimates track the particles."""
    import workloads as W
    a = W.config4(6)
    b = W.config4(6, particles=False)
    for (ca, P), (cb, rel) in zip(a["scenarios"], b["scenarios"]):
        assert ca == cb
        n = len(P["h"])
        assert abs(W.release_particle_estimate(rel, b["dx"]) - n) <= 0.02 * n
