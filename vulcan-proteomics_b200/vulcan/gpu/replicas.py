"""Replicas across GPUs: the search partitions by run (and by spectrum) with no exchange, so N GPUs each hold the
index and search their own runs; the only collectives are for the report (the slowest rank's time, totals) and,
when asked for, the all-gather of the finished PSM tables (host objects, after the search).  One process per GPU,
torch.distributed for the plumbing (NCCL on GPUs, gloo on CPU)."""
from __future__ import annotations

import torch
import torch.distributed as dist


def shard_runs(runs: list, rank: int, world: int) -> list:
    """The runs of this rank: whole runs dealt round-robin by size (largest first), so ranks get similar work."""
    order = sorted(range(len(runs)), key=lambda i: -len(runs[i]))
    load = [0] * world
    mine = []
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        load[r] += len(runs[i])
        if r == rank:
            mine.append(i)
    return sorted(mine)


def max_over_ranks(x: float, device=None) -> float:
    """The largest value over the ranks (the job's elapsed time is the slowest rank's)."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, device=None) -> float:
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def _world():
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def search_runs(runs: list, search_many, gather: bool = False) -> list:
    """Many runs searched by every rank of the process group, each rank its shard (``shard_runs``) through
    ``search_many(list of runs) -> [(table, stats), ...]`` (e.g. ``engine.Searcher.search_many``).  Returns
    [(run index, table, stats)] of this rank's runs in run order, or with ``gather`` every run's result on every rank
    (an all-gather of the finished tables as host objects).  Without a process group: all runs, this process."""
    rank, world = _world()
    mine = shard_runs(runs, rank, world)
    res = search_many([runs[i] for i in mine]) if mine else []
    out = [(i, t, st) for i, (t, st) in zip(mine, res)]
    if gather and world > 1:
        parts = [None] * world
        dist.all_gather_object(parts, out)
        out = sorted((x for part in parts for x in part), key=lambda x: x[0])
    return out
