"""Job sharding across GPUs: one process per GPU, no data-path collective.

Sweeps, batches and served streams are independent jobs (the reference runs
them one orf.fdtd2D call at a time: examples/cpo_box_scan.m:23-31,
optimizeGratingCoupler.m:1-12).  Across GPUs they are partitioned by cost
(cells x steps, greedy longest-first onto the least-loaded rank); every rank
runs its share through the batched engine on its own GPU, and the results
are gathered once on the host (torch.distributed all_gather_object over the
process group: NCCL on GPUs, gloo on CPU).  A single job is never split: one
C1-C3 job fits one GPU, so more GPUs mean more jobs at once ("replicas").
"""
from __future__ import annotations

from typing import Callable, Sequence


def partition_by_cost(costs: Sequence[float], world: int) -> list[list[int]]:
    """Indices of the jobs each of `world` ranks runs (longest first onto the
    least-loaded rank; ties go to the lower rank).  Every index appears once."""
    if world < 1:
        raise ValueError("world must be >= 1")
    loads = [0.0] * world
    shares: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda q: (-float(costs[q]), q)):
        r = min(range(world), key=lambda w: (loads[w], w))
        shares[r].append(i)
        loads[r] += float(costs[i])
    return [sorted(s) for s in shares]


def sharded_map(run_batch: Callable[[list], list], items: Sequence, costs: Sequence[float], group=None) -> list:
    """run_batch(items[share]) on every rank's share; returns all results in
    the order of `items` on every rank.  Without an initialised process group
    it is run_batch(items)."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return list(run_batch(list(items)))
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    share = partition_by_cost(costs, world)[rank]
    mine = list(run_batch([items[i] for i in share])) if share else []
    if len(mine) != len(share):
        raise RuntimeError("run_batch returned a wrong number of results")
    gathered: list = [None] * world
    dist.all_gather_object(gathered, list(zip(share, mine)), group=group)
    out: list = [None] * len(items)
    for part in gathered:
        for i, r in part:
            out[i] = r
    return out
