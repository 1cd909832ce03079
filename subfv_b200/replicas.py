"""Host-side logic of running the path on several GPUs of one node, one process per GPU.

The path does not shard inside one domain (one mesh per GPU, as the reference's MPI
decomposition is not used on the device), so several GPUs run independent work: whole
replicas of a benchmark, or disjoint subsets of independent problems (shock tubes,
serving requests). There is no data-path collective; the only exchanges are the
timing and counting reductions here, over torch.distributed (NCCL on GPUs, gloo on CPU).
"""
from __future__ import annotations

import heapq


def _dist():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        return dist
    return None


def _tensor(values, device):
    import torch
    return torch.tensor(values, dtype=torch.float64, device=device)


def _device():
    import torch
    import torch.distributed as dist
    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def max_over_ranks(x: float) -> float:
    """The largest of the ranks' values (the timing rule: the slowest rank's time)."""
    dist = _dist()
    if dist is None:
        return float(x)
    t = _tensor([x], _device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_throughput(units: float, seconds: float) -> tuple[float, float]:
    """Whole-job throughput of independent work: the units all ranks processed over the
    slowest rank's time. Returns (units per second, max seconds)."""
    dist = _dist()
    if dist is None:
        return units / seconds, seconds
    t = _tensor([units, seconds], _device())
    u = t[:1].clone()
    s = t[1:].clone()
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    dist.all_reduce(s, op=dist.ReduceOp.MAX)
    return float(u.item()) / float(s.item()), float(s.item())


def partition_by_cells(cells: list[int], world: int) -> list[list[int]]:
    """Split problems over `world` ranks by cell count: largest first, each to the least
    loaded rank (ties to the lower rank); each rank's list keeps the original order.
    Deterministic, so every rank computes the same partition without communication."""
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0, r) for r in range(world)]
    owner = [0] * len(cells)
    for i in sorted(range(len(cells)), key=lambda k: (-cells[k], k)):
        load, r = heapq.heappop(heap)
        owner[i] = r
        heapq.heappush(heap, (load + cells[i], r))
    return [[i for i in range(len(cells)) if owner[i] == r] for r in range(world)]


def gather_lists(local: list) -> list:
    """Concatenation of every rank's list, rank order (e.g. per-request latencies)."""
    dist = _dist()
    if dist is None:
        return list(local)
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, list(local))
    return [x for part in out for x in part]


def run_partitioned(sizes: list[int], solve):
    """Independent problems over the ranks: partition_by_cells on their sizes, each rank
    solves its share with solve(indices) -> (one result per index, units processed,
    seconds), then every rank receives all results in problem order. Returns (results,
    whole-job units per second, the slowest rank's seconds). With one process it is
    solve(all problems)."""
    dist = _dist()
    world = dist.get_world_size() if dist else 1
    rank = dist.get_rank() if dist else 0
    mine = partition_by_cells(list(sizes), world)[rank]
    results, units, seconds = solve(mine)
    if len(results) != len(mine):
        raise ValueError("solve must return one result per problem index")
    rate, slowest = aggregate_throughput(float(units), float(seconds))
    out = [None] * len(sizes)
    for i, r in gather_lists(list(zip(mine, results))):
        out[i] = r
    return out, rate, slowest
