"""Multi-GPU plumbing for KIFMM evaluation: independent units, no data-path collective.

One FMM instance does not shard (a locally-essential-tree ghost exchange
would be needed; the reference has none), so several GPUs are used in two
ways, both without any collective on the data path:

* replicas -- every rank evaluates its own copy of the workload (bench.py);
* instance sharding -- many independent FMM instances (the batched
  workload) are split over ranks by greedy longest-processing-time on an
  estimated cost, and each rank evaluates its own instances.

torch.distributed (NCCL on GPUs, gloo on CPU) is used only for the barrier
around the timed region and the max-over-ranks reduction of times.
"""
from __future__ import annotations

import heapq
import math


def estimated_cost(n_points: int, np_: int = 6, sdof: int = 1, ptsmax: int = 64) -> float:
    """Relative cost of one eval: near field (~n * 27 * ptsmax/2 interactions)
    plus the V list (~n/ptsmax * 8 * 189 pairs * nfreq), in arbitrary units."""
    nfreq = (2 * np_) ** 2 * (np_ + 1)
    near = n_points * 27.0 * ptsmax / 2.0
    far = (n_points / max(1, ptsmax)) * 8.0 * 189.0 * nfreq * sdof * 0.5
    return near + far


def lpt_partition(costs, nranks: int):
    """Greedy longest-processing-time: instances in decreasing cost order, each
    to the currently least-loaded rank.  Returns one sorted index list per rank."""
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    heap = [(0.0, r) for r in range(nranks)]
    heapq.heapify(heap)
    parts = [[] for _ in range(nranks)]
    for i in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(p) for p in parts]


def imbalance(costs, parts) -> float:
    """max rank load / mean rank load (1.0 = perfect)."""
    loads = [sum(costs[i] for i in p) for p in parts]
    mean = sum(loads) / len(loads) if loads else 0.0
    return max(loads) / mean if mean > 0 else 1.0


def instance_cost(inst, np_: int = 6, ptsmax: int = 64) -> float:
    """estimated_cost of one batched instance (a workloads.batched_instances
    entry): the source dofs of its equivalent kernel weigh the V list (4 for
    Stokes through kernel 301, 1 for Laplace)."""
    sdof_mm = 4 if inst["kt"] in (311, 321) else 3 if inst["kt"] in (511, 521) else 1
    return estimated_cost(inst["n"], np_, sdof_mm, ptsmax)


def shard_instances(insts, rank: int, world: int):
    """This rank's share of independent FMM instances: the indices of its
    longest-processing-time part (sorted) and the partition's imbalance
    (max rank load / mean rank load)."""
    if not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    costs = [instance_cost(i) for i in insts]
    parts = lpt_partition(costs, world)
    return parts[rank], imbalance(costs, parts)


def batched_run(insts, rank: int, world: int, run_shard, rhs: int = 1, dist=None, device=None):
    """Evaluates a rank's share of independent instances and combines the
    ranks' timings: run_shard(indices) sets up and times this rank's
    instances and returns (ms per step, extra); the step time is the max over
    ranks (no collective touches the data).  Returns a dict with the whole-job
    Mpoints/s (every instance's points x rhs over the slowest rank's time),
    the max time, this rank's indices, the imbalance and extra."""
    mine, imb = shard_instances(insts, rank, world)
    ms, extra = run_shard(mine)
    ms = reduce_max(ms, dist, device)
    npts = sum(int(i["n"]) for i in insts)
    return {"value": npts * rhs / (ms / 1e3) / 1e6 if ms > 0 else float("nan"), "ms": ms, "mine": mine,
            "imbalance": imb, "extra": extra}


def reduce_max(value: float, dist=None, device=None) -> float:
    """Max of a float over all ranks (identity without a process group)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(value: float, dist=None, device=None) -> float:
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def weak_scaling_value(points_per_rank: int, world: int, max_ms: float) -> float:
    """Whole-job Mpoints/s: all ranks' points over the slowest rank's time."""
    if max_ms <= 0 or math.isnan(max_ms):
        return float("nan")
    return world * points_per_rank / (max_ms / 1e3) / 1e6
