"""Multi-GPU plumbing for the packing workload.

Packing runs on different trays share nothing, so the path shards by tray with
no data-path collective: rank r packs trays r, r+world, r+2*world, ... (or, in
the benchmark, its own seeded item stream).  The only collectives are the
timing and count reductions around a timed region (max of the device time over
ranks, sum of placed items), done with torch.distributed on whatever backend
the caller initialised (NCCL on GPUs, gloo in the CPU tests).
"""
from __future__ import annotations

from typing import List, Sequence, Tuple


def tray_shard(n_trays: int, rank: int, world: int) -> List[int]:
    """Indices of the trays rank `rank` packs (round robin)."""
    if world <= 0 or not (0 <= rank < world):
        raise ValueError(f"bad rank {rank} for world size {world}")
    return list(range(rank, n_trays, world))


def stream_seed(rank: int, base: int = 1) -> int:
    """Seed of rank `rank`'s independent item stream (weak scaling)."""
    return base + 1000 * rank


def reduce_run(local_ms: float, local_items: float, device=None) -> Tuple[float, float]:
    """(max over ranks of local_ms, sum over ranks of local_items); identity
    when torch.distributed is not initialised."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(local_ms), float(local_items)
    t = torch.tensor([local_ms], dtype=torch.float64, device=device)
    c = torch.tensor([local_items], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return float(t.item()), float(c.item())


def balanced_order(costs: Sequence[float], world: int) -> List[List[int]]:
    """Greedy longest-first assignment of trays with estimated costs to ranks
    (for uneven tray sizes); returns per-rank index lists."""
    loads = [0.0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: -costs[k]):
        r = min(range(world), key=lambda q: loads[q])
        out[r].append(i)
        loads[r] += costs[i]
    return out
