"""Multi-rank helpers: replica throughput aggregation and scene-to-rank assignment.

The particle-fluid path has no exchange step between independent scenes, so
multi-GPU runs either replicate one scene per rank or shard a list of
independent scenes across ranks; neither needs a collective on the data path.
Only the final timing / statistics are combined (max of device times, sum of
work), over whatever process group the caller initialised (NCCL on GPUs,
gloo in the CPU tests).
"""
from __future__ import annotations

import heapq


def aggregate_throughput(local_units: float, local_ms: float, group=None) -> tuple[float, float]:
    """(units summed over ranks, max device milliseconds over ranks)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(local_units), float(local_ms)
    backend = dist.get_backend(group)
    dev = torch.device("cuda") if backend == "nccl" else torch.device("cpu")
    units = torch.tensor([float(local_units)], dtype=torch.float64, device=dev)
    ms = torch.tensor([float(local_ms)], dtype=torch.float64, device=dev)
    dist.all_reduce(units, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(ms, op=dist.ReduceOp.MAX, group=group)
    return float(units.item()), float(ms.item())


def lpt_assign(costs, n_ranks: int) -> list[list[int]]:
    """Longest-processing-time-first assignment of items (by cost) to ranks.

    Returns, per rank, the item indices in descending cost order; ties are
    broken by item index so every rank computes the same assignment.
    """
    if n_ranks < 1:
        raise ValueError("n_ranks must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(n_ranks)]
    heapq.heapify(heap)
    out = [[] for _ in range(n_ranks)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return out
