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


RECORD_BYTES = 32   # PSB_SHARD_RECORD_BYTES: one rank's decision (score, found, orientation, x, y, z)

ExchangeFn = None   # ctypes type of psb_exchange_fn, made on first use


def _exchange_type():
    import ctypes
    global ExchangeFn
    if ExchangeFn is None:
        ExchangeFn = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p)
    return ExchangeFn


def nccl_exchange(local, gathered, stream):
    """The exchange of psb_pack_staged_sharded over the initialised process
    group: an all-gather of every rank's decision record, queued on the
    engine's stream.  local: uint8 tensor of RECORD_BYTES, gathered: uint8
    tensor of world * RECORD_BYTES, both on this rank's GPU."""
    import torch
    import torch.distributed as dist

    def cb(_ctx):
        try:
            with torch.cuda.stream(stream):
                dist.all_gather_into_tensor(gathered, local)
            return 0
        except Exception:  # noqa: BLE001  (reported as the engine's error)
            return 1
    return _exchange_type()(cb)


class InProcessExchange:
    """The exchange for `world` ranks running as threads of one process, each
    with its own tray and stream on the same or different GPUs (used to run
    the sharded loop where fewer GPUs than ranks are available).  Per item
    every rank waits for its own stream, publishes its record on the host,
    waits for the others (a host barrier with a timeout, no device-side
    wait), and copies all records into its gathered buffer on its stream."""

    def __init__(self, world: int, timeout: float = 120.0):
        import threading
        self.world = world
        self.recs = [None] * world
        self.barrier = threading.Barrier(world, timeout=timeout)

    def callback(self, rank, local, gathered, stream):
        import torch

        def cb(_ctx):
            try:
                stream.synchronize()
                self.recs[rank] = local.cpu()
                self.barrier.wait()
                with torch.cuda.stream(stream):
                    gathered.copy_(torch.cat(self.recs).to(gathered.device))
                stream.synchronize()
                self.barrier.wait()
                return 0
            except Exception:  # noqa: BLE001
                self.barrier.abort()
                return 1
        return _exchange_type()(cb)


def pack_sharded_on_device(items, tray_size, num_orientations: int = 24, interlocking_free: bool = False,
                           sort_by_volume: bool = True, rank: int = 0, world: int = 1, exchange=None,
                           device=None):
    """One rank of the orientation-sharded greedy loop on the device
    (psb_pack_staged_sharded): this rank searches orientations o with
    o % world == rank, decisions are exchanged per item by `exchange` (a
    callable (local, gathered, stream) -> ctypes callback; None with world
    == 1) and every rank places the merged winner.  Returns (final tray,
    per-item (success, position, orientation, score)) in the items' original
    order, identical on every rank and to BinPacker(...).pack_voxels(items)."""
    import ctypes

    import numpy as np
    import torch

    from .proposal import PsbResult, check, lib
    from .rotations import orientation_maps

    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    maps = np.ascontiguousarray(orientation_maps(num_orientations), np.int32)
    arrs = [np.ascontiguousarray(np.asarray(i, dtype=np.int32)) for i in items]
    vols = [int(np.count_nonzero(a > 0)) for a in arrs]
    order = list(np.argsort(vols)[::-1]) if sort_by_volume else list(range(len(arrs)))
    seq = [arrs[k] for k in order]
    L = lib()
    vp = ctypes.c_void_p
    L.psb_tray_set.argtypes = [vp, vp, vp]
    L.psb_pack_stage.argtypes = [vp, vp, vp, ctypes.c_int]
    L.psb_pack_staged_sharded.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int32, ctypes.c_int,
                                          ctypes.c_int, vp, vp, vp, vp, vp, vp]
    L.psb_tray_stream.argtypes = [vp, vp]
    t = ctypes.c_void_p()
    check(L.psb_tray_create(*[int(d) for d in tray_size], ctypes.byref(t)))
    tray = np.zeros(tuple(int(d) for d in tray_size), np.int32)
    res = (PsbResult * len(seq))()
    try:
        with torch.cuda.device(dev):
            local = torch.zeros(RECORD_BYTES, dtype=torch.uint8, device=dev)
            gathered = torch.zeros(RECORD_BYTES * world, dtype=torch.uint8, device=dev)
            sp = ctypes.c_void_p()
            check(L.psb_tray_stream(t, ctypes.byref(sp)))
            stream = torch.cuda.ExternalStream(sp.value, device=dev)
            cb = exchange(local, gathered, stream) if exchange is not None else None
            check(L.psb_tray_set(t, tray.ctypes.data, None))
            ptrs = (ctypes.c_void_p * len(seq))(*[a.ctypes.data for a in seq])
            dims = np.ascontiguousarray(np.array([a.shape for a in seq], np.int32).ravel())
            check(L.psb_pack_stage(t, ptrs, dims.ctypes.data, len(seq)))
            torch.cuda.synchronize(dev)
            check(L.psb_pack_staged_sharded(t, maps.ctypes.data, len(maps), 1 if interlocking_free else 0, 0,
                                            rank, world, local.data_ptr(), gathered.data_ptr(),
                                            ctypes.cast(cb, vp) if cb is not None else None, None, res,
                                            tray.ctypes.data))
    finally:
        L.psb_tray_destroy(t)
    out = [None] * len(arrs)
    for r, k in zip(res, order):
        out[k] = (True, (r.x, r.y, r.z), r.orientation, r.score) if r.found else (False, None, 0, None)
    return tray, out


def pack_orientation_sharded(items, tray_size, num_orientations: int = 24, interlocking_free: bool = False,
                             sort_by_volume: bool = True, device=None):
    """Pack one tray with its orientations spread over the ranks of the
    initialised process group (one GPU per rank, NCCL; a single process when
    none): the device-resident loop with the candidate pre-filter, one
    decision record all-gathered per item.  Returns (final tray, per-item
    (success, position, orientation, score)) in the items' original order;
    identical on every rank and to BinPacker(...).pack_voxels(items)."""
    import torch.distributed as dist

    rank, world = 0, 1
    if dist.is_available() and dist.is_initialized():
        rank, world = dist.get_rank(), dist.get_world_size()
    return pack_sharded_on_device(items, tray_size, num_orientations, interlocking_free, sort_by_volume, rank,
                                  world, nccl_exchange if world > 1 else None, device)


def pack_sharded_protocol(items, tray_size, num_orientations, interlocking_free, search, place, exchange,
                          rank: int, world: int, sort_by_volume: bool = True):
    """The sharded loop's host protocol with the search and the placement
    supplied by the caller (the oracle in the CPU tests): per item in packing
    order this rank searches its orientations, the ranks' records are
    exchanged (exchange(local) -> merged record) and the winner is placed.
    search(tray, item, orientations) -> (found, score, orientation, x, y, z)
    with the global orientation index; place(tray, item, orientation, pos,
    item_id) -> new tray.  Returns (tray, per-item records in search order)."""
    import numpy as np
    arrs = [np.asarray(i, dtype=np.int32) for i in items]
    vols = [int(np.count_nonzero(a > 0)) for a in arrs]
    order = list(np.argsort(vols)[::-1]) if sort_by_volume else list(range(len(arrs)))
    mine = orientation_shard(num_orientations, rank, world)
    tray = np.zeros(tuple(int(d) for d in tray_size), np.int32)
    placed, recs = 0, []
    for k in order:
        local = search(tray, arrs[k], mine) if mine else (0, 0.0, -1, -1, -1, -1)
        rec = exchange(local)
        if rec[0]:
            placed += 1
            tray = place(tray, arrs[k], int(rec[2]), (int(rec[3]), int(rec[4]), int(rec[5])), placed)
        recs.append(tuple(rec))
    return tray, recs
