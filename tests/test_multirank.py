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
