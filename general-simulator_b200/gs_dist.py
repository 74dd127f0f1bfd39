"""Multi-GPU plumbing of the phase-field step: replicas only.

A single simulation fits one B200 (603 MB at 256^3 x 3 variants, FP32), so
nothing here splits a grid.  What shards is the ensemble: independent
simulations are dealt to ranks (one process per GPU) by a cost model, each
rank advances its share as one gs_batch with no collective during stepping,
and the per-simulation statistics are gathered on the host at the end.  The
only collectives are the host gather and the max-over-ranks timing, both
through torch.distributed (NCCL on GPUs, gloo in the CPU tests).
"""
from __future__ import annotations

import math
from typing import Dict, List, Sequence

import gs_b200 as gb


def sim_cost(p: gb.GsParams) -> float:
    """Relative cost of one step: V N log2 N (five FFT-bound sweeps)."""
    n = p.nx * p.ny * p.nz
    return p.nvariants * n * max(math.log2(n), 1.0)


def shard(costs: Sequence[float], world: int) -> List[List[int]]:
    """Deal items to `world` ranks, largest first to the least loaded rank
    (longest-processing-time rule); ties go to the lower rank.  Returns the
    item indices of every rank, each list in increasing order."""
    if world < 1:
        raise ValueError("world size must be >= 1")
    load = [0.0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(i)
        load[r] += costs[i]
    return [sorted(x) for x in out]


def my_share(params: Sequence[gb.GsParams], rank: int, world: int) -> List[int]:
    return shard([sim_cost(p) for p in params], world)[rank]


def gather_stats(local: Dict[int, dict], world: int) -> Dict[int, dict]:
    """Merge every rank's {sim index: stats} into one dict on every rank."""
    if world == 1:
        return dict(local)
    import torch.distributed as dist

    parts: list = [None] * world
    dist.all_gather_object(parts, local)
    merged: Dict[int, dict] = {}
    for part in parts:
        for k, v in part.items():
            if k in merged:
                raise RuntimeError(f"simulation {k} reported by two ranks")
            merged[k] = v
    return merged


def max_over_ranks(x: float, world: int, device: str = "cpu") -> float:
    """The largest value over ranks (device time of the slowest rank)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_ensemble_shard(params: Sequence[gb.GsParams], eta0: Sequence, rank: int, world: int, nsteps: int,
                       use_graph: bool = True, gather: bool = True) -> Dict[int, dict]:
    """Advance this rank's share of the ensemble nsteps steps as one batch
    and return the gathered statistics of every simulation (all ranks), or
    only this rank's with gather=False."""
    mine = my_share(params, rank, world)
    local: Dict[int, dict] = {}
    if mine:
        b = gb.Batch([params[i] for i in mine])
        try:
            for j, i in enumerate(mine):
                b.set_eta(j, eta0[i])
            b.use_graph(use_graph)
            b.step(nsteps)
            for j, i in enumerate(mine):
                local[i] = b.stats(j)
        finally:
            b.close()
    return gather_stats(local, world) if gather else local
