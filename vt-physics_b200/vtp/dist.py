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


def scene_cost(scene) -> float:
    """Relative cost of one substep of a scene: fluid particles, times 2 for the pressure-solved
    schemes (DFSPH / IMM run about twice as many neighbour passes as PBF's 4 iterations)."""
    return scene.n_fluid * (1.0 if scene.solver == "PBF" else 2.0)


def scene_share(scenes, n_ranks: int, rank: int) -> list[int]:
    """Indices of the scenes rank `rank` advances (LPT on scene_cost), ascending."""
    return sorted(lpt_assign([scene_cost(s) for s in scenes], n_ranks)[rank])


def gather_scene_results(local: dict, group=None) -> dict:
    """Merge every rank's {scene index: result} (any picklable result) on every rank.  The
    only exchange of a sharded batch, once, after the run."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return dict(local)
    parts = [None] * dist.get_world_size(group)
    dist.all_gather_object(parts, local, group=group)
    out = {}
    for p in parts:
        overlap = set(out) & set(p)
        if overlap:
            raise RuntimeError(f"scenes {sorted(overlap)} were advanced by more than one rank")
        out.update(p)
    return out
