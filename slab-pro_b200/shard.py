"""Scenario sharding across GPUs: one process per GPU, each running its own
batch of whole scenarios on a copy of the shared terrain.

Release scenarios are independent (the reference runs one per process,
src/main.cpp:29-57), so an ensemble shards by scenario with no collective on
the data path: every rank computes the same deterministic assignment, runs
its share as one slab_batch, and the host gathers the per-scenario results
(a gather of small Python objects, gloo or NCCL) at the end.

The assignment balances the estimated work (particles x simulated time) with
the longest-processing-time rule and keeps every rank's estimated device
footprint under its memory budget.
"""
from __future__ import annotations

from typing import Callable, Sequence

# device bytes per particle of the FP32 split path: two particle buffers
# (cell, offset, velocity, h, m, id, vz, z: 40 B each) and binning temporaries
BYTES_PER_PARTICLE = 2 * 40 + 48
# device bytes per node of a scenario's node blocks (velocity + FLIP 16,
# maxima 8, output fields 20) and its share of the P2G partials
BYTES_PER_NODE = 44 + 30


def footprint_bytes(n_particles: int, nodes_estimate: int | None = None) -> int:
    """Estimated device memory of one scenario: its particles and the node
    blocks its flow touches (by default four nodes per particle, the spread
    of a developed flow)."""
    nodes = 4 * n_particles if nodes_estimate is None else nodes_estimate
    return BYTES_PER_PARTICLE * n_particles + BYTES_PER_NODE * nodes


def assign(costs: Sequence[float], world: int, footprints: Sequence[int] | None = None,
           budget_bytes: int | None = None) -> list[list[int]]:
    """Scenario indices per rank. Longest processing time first: scenarios in
    decreasing cost (ties by index) go to the rank with the least cost so far
    (ties by rank), skipping ranks whose footprint would exceed budget_bytes.
    Deterministic, so every rank computes the same assignment on its own.
    Raises ValueError if a scenario fits no rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    n = len(costs)
    fp = list(footprints) if footprints is not None else [0] * n
    if len(fp) != n:
        raise ValueError("one footprint per scenario")
    load = [0.0] * world
    used = [0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(n), key=lambda k: (-float(costs[k]), k)):
        ranks = sorted(range(world), key=lambda r: (load[r], r))
        for r in ranks:
            if budget_bytes is None or used[r] + fp[i] <= budget_bytes:
                out[r].append(i)
                load[r] += float(costs[i])
                used[r] += fp[i]
                break
        else:
            raise ValueError(f"scenario {i} ({fp[i]} bytes) fits on no rank within {budget_bytes} bytes")
    for lst in out:
        lst.sort()
    return out


def run_sharded(scenarios: Sequence, rank: int, world: int, cost: Callable, run_batch: Callable,
                footprint: Callable | None = None, budget_bytes: int | None = None, gather: Callable | None = None):
    """Run this rank's share of `scenarios` with run_batch(list of (index,
    scenario)) -> {index: result}, then gather: returns (the full
    {index: result} on rank 0 -- None elsewhere -- when gather is given, else
    this rank's results; the assignment). gather(obj) must return the list of
    every rank's obj on rank 0 (torch.distributed.gather_object)."""
    costs = [cost(s) for s in scenarios]
    fps = [footprint(s) for s in scenarios] if footprint else None
    shards = assign(costs, world, fps, budget_bytes)
    mine = run_batch([(i, scenarios[i]) for i in shards[rank]])
    if gather is None:
        return mine, shards
    parts = gather(mine)
    if parts is None:
        return None, shards
    merged = {}
    for p in parts:
        merged.update(p)
    return merged, shards


def torch_gather(group=None) -> Callable:
    """gather for run_sharded over torch.distributed (the default process
    group): rank 0 gets every rank's object."""
    import torch.distributed as dist

    def g(obj):
        world = dist.get_world_size(group)
        out = [None] * world if dist.get_rank(group) == 0 else None
        dist.gather_object(obj, out, dst=0, group=group)
        return out

    return g
