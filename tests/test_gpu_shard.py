"""The orientation-sharded device loop (psb_pack_staged_sharded) against the
oracle's golden traces.

Every call of this suite gets one GPU, so the ranks run as threads of one
process, each with its own tray and stream on that GPU, and exchange their
per-item decision records on the host (InProcessExchange: a host barrier with
a timeout; no kernel waits on another).  The device loop, the per-rank
orientation subsets, the record layout and the merge are the ones a
multi-GPU run uses with NCCL (nccl_exchange); only the transport differs.
"""
import threading

import numpy as np
import pytest

from oracle.trace_replay import load_trace, trace_items

pytestmark = pytest.mark.gpu


def _ranks(name, world):
    import torch
    from psacking_b200.shard import InProcessExchange, pack_sharded_on_device
    tr = load_trace(name)
    seq = trace_items(tr)
    ex = InProcessExchange(world)
    out, errs = [None] * world, []

    def work(r):
        try:
            torch.cuda.set_device(0)
            out[r] = pack_sharded_on_device(seq, tuple(tr["tray"]), tr["num_orientations"], tr["interlocking_free"],
                                            sort_by_volume=False, rank=r, world=world,
                                            exchange=lambda l, g, s: ex.callback(r, l, g, s))
        except Exception as e:  # noqa: BLE001
            errs.append(e)
    th = [threading.Thread(target=work, args=(r,)) for r in range(world)]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=600)
    assert not errs, errs
    return tr, out


@pytest.mark.parametrize("name,world", [("config3_seed1", 2), ("config2_seed0", 3), ("config1_seed3", 1)])
def test_sharded_loop_matches_trace(gpu_core, name, world):
    import hashlib
    tr, out = _ranks(name, world)
    for tray, recs in out:
        got = [[1, *pos, o, sc] if f else [0, -1, -1, -1, 0, 0.0] for f, pos, o, sc in recs]
        bad = [i for i, (a, b) in enumerate(zip(got, tr["records"])) if a != b]
        assert not bad, (bad[0], got[bad[0]], tr["records"][bad[0]])
        assert hashlib.sha256(np.ascontiguousarray(tray).tobytes()).hexdigest() == tr["tray_sha256"]


def test_sharded_loop_single_process_group(gpu_core):
    """Without a process group pack_orientation_sharded is the world-1 loop."""
    from psacking_b200.shard import pack_orientation_sharded
    tr = load_trace("config1_seed5")
    seq = trace_items(tr)
    tray, recs = pack_orientation_sharded(seq, tuple(tr["tray"]), 1, False, sort_by_volume=False)
    got = [[1, *pos, o, sc] if f else [0, -1, -1, -1, 0, 0.0] for f, pos, o, sc in recs]
    assert got == tr["records"]
