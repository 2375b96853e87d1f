"""Replica plumbing for multi-GPU runs.

The time-stepping path does not shard across GPUs in this build (the reference
is a single-domain, single-device model): N GPUs run N independent replicas or
disjoint subsets of an ensemble.  torch.distributed is used only for barriers
and for the max-over-ranks timing reduction -- never on the data path.
"""
from __future__ import annotations

from typing import List, Sequence


def partition(n_items: int, world: int, rank: int) -> List[int]:
    """Contiguous, balanced split of item indices [0, n_items) over ranks."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad world/rank")
    base, extra = divmod(n_items, world)
    start = rank * base + min(rank, extra)
    stop = start + base + (1 if rank < extra else 0)
    return list(range(start, stop))


def partition_by_cost(costs: Sequence[float], world: int, rank: int) -> List[int]:
    """Greedy longest-processing-time split of weighted items (e.g. cell counts)."""
    loads = [0.0] * world
    owner = {}
    for i in sorted(range(len(costs)), key=lambda k: -costs[k]):
        r = min(range(world), key=lambda k: loads[k])
        owner[i] = r
        loads[r] += costs[i]
    return sorted(i for i, r in owner.items() if r == rank)


def _dist():
    import torch.distributed as dist

    return dist if dist.is_available() and dist.is_initialized() else None


def barrier() -> None:
    d = _dist()
    if d is not None:
        d.barrier()


def allreduce_max(x: float) -> float:
    """Max of a scalar over all ranks (works with the gloo and nccl backends)."""
    d = _dist()
    if d is None:
        return float(x)
    import torch

    dev = "cuda" if d.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    d.all_reduce(t, op=d.ReduceOp.MAX)
    return float(t.item())


def allreduce_sum(x: float) -> float:
    d = _dist()
    if d is None:
        return float(x)
    import torch

    dev = "cuda" if d.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    d.all_reduce(t, op=d.ReduceOp.SUM)
    return float(t.item())
