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


# --------------------------------------------------------------------------
# orientation sharding of one tray
# --------------------------------------------------------------------------
# Every rank holds the whole tray, its distance field and spectra.  For each
# item, rank r searches the orientations o with o % world == r, exchanges one
# small decision record (found, score, orientation, x, y, z) with the others,
# and every rank applies the same winner: the smallest score, and on equal
# scores the lowest orientation index, which is the reference's strict <
# over the orientations in order (fft3.cu:1625, packer.py:500).  Within an
# orientation the exact search's own tie rule already picked the position.
# The trays therefore stay identical on every rank without being exchanged.

def orientation_shard(n_orient: int, rank: int, world: int) -> List[int]:
    """Global orientation indices rank `rank` searches."""
    if world <= 0 or not (0 <= rank < world):
        raise ValueError(f"bad rank {rank} for world size {world}")
    return list(range(rank, n_orient, world))


def merge_decisions(records: Sequence[Tuple]) -> Tuple:
    """records: per rank (found, score, orientation, x, y, z) with the global
    orientation index.  The winner over all ranks (found = 0 when none)."""
    best = None
    for r in records:
        found, score, orient = int(r[0]), float(r[1]), int(r[2])
        if not found:
            continue
        if best is None or score < best[1] or (score == best[1] and orient < best[2]):
            best = (1, score, orient, int(r[3]), int(r[4]), int(r[5]))
    return best if best is not None else (0, 0.0, -1, -1, -1, -1)


def exchange_decision(local: Tuple, device=None) -> Tuple:
    """All-gather the ranks' decision records (one float64 tensor of 6 values
    per rank, exact for scores and indices) and merge them; identity without
    an initialised process group."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return merge_decisions([local])
    t = torch.tensor([float(v) for v in local], dtype=torch.float64, device=device)
    out = [torch.empty_like(t) for _ in range(dist.get_world_size())]
    dist.all_gather(out, t)
    return merge_decisions([tuple(o.tolist()) for o in out])


def pack_orientation_sharded(items, tray_size, num_orientations: int = 24, interlocking_free: bool = False,
                             sort_by_volume: bool = True, device=None):
    """Pack one tray with its orientations spread over the ranks of the
    initialised process group (one GPU per rank; a single process when none).
    Returns (final tray, per-item (success, position, orientation, score)) in
    the items' original order; identical on every rank and to
    BinPacker(...).pack_voxels(items)."""
    import ctypes

    import numpy as np
    import torch.distributed as dist

    from .proposal import PsbResult, check, lib
    from .rotations import apply_map, orientation_maps

    rank, world = 0, 1
    if dist.is_available() and dist.is_initialized():
        rank, world = dist.get_rank(), dist.get_world_size()
    maps = orientation_maps(num_orientations)
    mine = orientation_shard(num_orientations, rank, world)
    arrs = [np.asarray(i, dtype=np.int32) for i in items]
    vols = [int(np.count_nonzero(a > 0)) for a in arrs]
    order = list(np.argsort(vols)[::-1]) if sort_by_volume else list(range(len(arrs)))
    L = lib()
    vp = ctypes.c_void_p
    L.psb_tray_search.argtypes = [vp, vp, vp, ctypes.c_int, ctypes.c_int, vp, vp]
    L.psb_tray_place.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                 ctypes.c_int, ctypes.c_int32]
    L.psb_tray_set.argtypes = [vp, vp, vp]
    L.psb_tray_get.argtypes = [vp, vp, vp]
    t = ctypes.c_void_p()
    check(L.psb_tray_create(*[int(d) for d in tray_size], ctypes.byref(t)))
    tray = np.zeros(tuple(int(d) for d in tray_size), np.int32)
    mode = (1 if (interlocking_free or num_orientations > 1) else 0) | (0x10 if interlocking_free else 0)
    out = [None] * len(arrs)
    placed = 0
    try:
        check(L.psb_tray_set(t, tray.ctypes.data, None))
        for k in order:
            ors = [np.ascontiguousarray(apply_map(arrs[k], maps[o])) for o in mine]
            local = (0, 0.0, -1, -1, -1, -1)
            if ors:
                ptrs = (ctypes.c_void_p * len(ors))(*[a.ctypes.data for a in ors])
                dims = np.ascontiguousarray(np.array([a.shape for a in ors], np.int32).ravel())
                r = PsbResult()
                check(L.psb_tray_search(t, ptrs, dims.ctypes.data, len(ors), mode, ctypes.byref(r), None))
                if r.found:
                    local = (1, r.score, mine[r.orientation], r.x, r.y, r.z)
            found, score, orient, x, y, z = exchange_decision(local, device=device)
            if found:
                it = np.ascontiguousarray(apply_map(arrs[k], maps[orient]))
                placed += 1
                check(L.psb_tray_place(t, it.ctypes.data, *it.shape, x, y, z, placed))
                out[k] = (True, (x, y, z), orient, score)
            else:
                out[k] = (False, None, 0, None)
        check(L.psb_tray_get(t, tray.ctypes.data, None))
    finally:
        L.psb_tray_destroy(t)
    return tray, out
