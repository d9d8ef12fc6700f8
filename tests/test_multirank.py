"""World-size-2 runs of the multi-GPU plumbing on CPU (gloo backend)."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from psacking_b200.shard import balanced_order, reduce_run, stream_seed, tray_shard


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        ms, items = reduce_run(10.0 + 5 * rank, 3 + rank)
        mine = tray_shard(7, rank, world)
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        seeds = [None] * world
        dist.all_gather_object(seeds, stream_seed(rank))
        q.put((rank, ms, items, gathered, seeds))
    finally:
        dist.destroy_process_group()


def test_two_rank_reduction_and_sharding():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, items, gathered, seeds in out:
        assert ms == 15.0           # max over ranks
        assert items == 7.0         # 3 + 4
        flat = sorted(i for g in gathered for i in g)
        assert flat == list(range(7))
        assert len(set(seeds)) == world


def test_single_process_identity():
    assert reduce_run(3.5, 2) == (3.5, 2.0)
    with pytest.raises(ValueError):
        tray_shard(4, 2, 2)


def test_balanced_order():
    parts = balanced_order([5, 1, 4, 2, 3], 2)
    assert sorted(i for p in parts for i in p) == [0, 1, 2, 3, 4]
    loads = [sum([5, 1, 4, 2, 3][i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= 1


def _merge_worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        from psacking_b200.shard import exchange_decision, orientation_shard
        mine = orientation_shard(24, rank, world)
        # each rank's local best over its own orientations, three cases:
        # a strict winner, an exact tie across ranks, nothing found anywhere
        cases = {
            "strict": (1, 120.0 - rank, mine[3], rank, 2, 0),
            "tie": (1, 55.0, mine[5], 7 + rank, 1, 0),
            "none": (0, 0.0, -1, -1, -1, -1),
        }
        res = {k: exchange_decision(v) for k, v in cases.items()}
        q.put((rank, mine, res))
    finally:
        dist.destroy_process_group()


def test_two_rank_orientation_sharding():
    """Orientation sharding of one tray: every orientation is searched by
    exactly one rank, and both ranks reach the same decision, with the
    reference's tie rule (equal scores: the lowest orientation index)."""
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_merge_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted([q.get(timeout=120) for _ in range(world)])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(o for _, mine, _ in out for o in mine) == list(range(24))
    (_, m0, r0), (_, m1, r1) = out
    assert r0 == r1
    assert r0["strict"] == (1, 119.0, m1[3], 1, 2, 0)          # rank 1 has the lower score
    assert r0["tie"] == (1, 55.0, min(m0[5], m1[5]), 7, 1, 0)  # lowest orientation index wins
    assert r0["none"] == (0, 0.0, -1, -1, -1, -1)


def test_merge_decisions_rules():
    from psacking_b200.shard import merge_decisions
    assert merge_decisions([(0, 0, -1, -1, -1, -1), (1, 3.0, 4, 1, 1, 1)]) == (1, 3.0, 4, 1, 1, 1)
    assert merge_decisions([(1, 3.0, 9, 0, 0, 0), (1, 3.0, 4, 1, 1, 1)])[2] == 4
    assert merge_decisions([(1, 2.0, 9, 0, 0, 0), (1, 3.0, 4, 1, 1, 1)])[2] == 9


def _oracle_search(interlock, n_orient):
    import numpy as np
    from oracle import psb_oracle as O

    def search(tray, item, mine):
        phi = O.calculate_distance(tray)
        ors = O.orientations(item, n_orient)
        best = (0, 0.0, -1, -1, -1, -1)
        for o in mine:
            r = np.ascontiguousarray(ors[o])
            if any(r.shape[a] > tray.shape[a] for a in range(3)):
                continue
            pos, found, sc = O.search_one(r, tray, phi, mode="block", interlock=interlock)
            if found and (not best[0] or sc < best[1]):   # strict <: the first in index order wins
                best = (1, sc, o, *pos)
        return best

    def place(tray, item, o, pos, item_id):
        r = np.ascontiguousarray(O.orientations(item, n_orient)[o])
        return O.place_in_tray(r, tray, pos, item_id)
    return search, place


def _loop_worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        import importlib.util
        from pathlib import Path
        from psacking_b200.shard import exchange_decision, pack_sharded_protocol
        spec = importlib.util.spec_from_file_location(
            "wl", Path(__file__).resolve().parent.parent / "psacking_b200" / "workloads.py")
        W = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(W)
        items = W.config1_items(4)[:6]
        search, place = _oracle_search(True, 6)
        tray, recs = pack_sharded_protocol(items, (30, 30, 14), 6, True, search, place, exchange_decision, rank, world)
        q.put((rank, tray, recs))
    finally:
        dist.destroy_process_group()


def test_two_rank_sharded_packing_loop():
    """The whole orientation-sharded packing loop at world size 2 (gloo):
    each rank searches its own orientations with the oracle, the decision
    records are all-gathered per item, and both ranks end with the same tray
    and the same placements as the unsharded oracle run."""
    import numpy as np
    from oracle import psb_oracle as O
    from oracle.trace_replay import load_workloads
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_loop_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted([q.get(timeout=300) for _ in range(world)], key=lambda x: x[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, t0, r0), (_, t1, r1) = out
    assert np.array_equal(t0, t1) and r0 == r1
    items = load_workloads().config1_items(4)[:6]
    want_tray, want = O.pack_voxels(items, (30, 30, 14), 6, True)
    assert np.array_equal(t0, want_tray)
    vols = [int((np.asarray(i) > 0).sum()) for i in items]
    order = list(np.argsort(vols)[::-1])
    for rec, k in zip(r0, order):
        w = want[k]
        assert bool(rec[0]) == w["success"]
        if w["success"]:
            assert (tuple(rec[3:6]), rec[2], rec[1]) == (w["position"], w["orientation_index"], w["score"])
