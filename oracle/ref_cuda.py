"""The reference's own cuFFT placement search, timed and recorded -- TEST
INFRASTRUCTURE ONLY (a measured baseline and a parity witness, never part of
the product path).

    python oracle/ref_cuda.py full   [--items N] [--out FILE]
    python oracle/ref_cuda.py sample --positions P1,P2,... [--out FILE]

Runs the reference's unmodified Python BinPacker (spectral_packer/packer.py)
over the reference's own pybind11 module, both built from the reference
sources by oracle/Makefile into oracle/_ref/ (sm_100a, cuFFT).  Needs a GPU.

full    packs the benchmark's item stream (240x123x100 tray, 350 config-3
        items of seed 1, 24 orientations, interlocking-free) from an empty
        tray in one BinPacker.pack_voxels call, as a user would; prints the
        wall time and every item's (found, x, y, z, orientation, score) in
        search order.
sample  replays the tray states of the oracle's trace of that stream
        (tests/golden/traces/config3_seed1.json) and times
        BinPacker.pack_voxels([item], initial_tray=state) for the item at
        each listed search position (one item searched in 24 orientations and
        placed, the unit of the benchmark's metric).
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent


def reference_packer():
    ref = HERE / "_ref"
    if not (ref / "spectral_packer" / "packer.py").exists():
        raise FileNotFoundError("oracle/_ref is not built (make -C oracle)")
    sys.path.insert(0, str(ref))
    import spectral_packer  # noqa: F401
    from spectral_packer import BinPacker, _core
    return BinPacker, _core


def run_full(n_items, out):
    from oracle.trace_replay import load_workloads, record
    BinPacker, core = reference_packer()
    W = load_workloads()
    items = W.config3_items(1, n=350)
    vols = [int(np.sum(i > 0)) for i in items]
    items = [items[i] for i in np.argsort(vols)[::-1]][:n_items]
    packer = BinPacker(W.TRAY3, num_orientations=24, interlocking_free=True)
    packer.pack_voxels(items[:1])  # CUDA context, cuFFT plans, module load
    # the module caches the tray context by a generation number that every
    # pack_voxels call restarts at 0 (bindings.cpp:209, 236-239): drop it
    core.gpu_tray_cleanup()
    t0 = time.perf_counter()
    res = packer.pack_voxels(items, sort_by_volume=False)
    dt = time.perf_counter() - t0
    recs = [record(p.success, p.position, p.orientation_index, p.score) for p in res.placements]
    doc = {"items": n_items, "seconds": dt, "items_per_s": n_items / dt, "num_placed": res.num_placed,
           "items_placed_per_s": res.num_placed / dt, "records": recs}
    Path(out).write_text(json.dumps(doc) + "\n")
    print(json.dumps({k: v for k, v in doc.items() if k != "records"}))


def run_sample(positions, out):
    from oracle.trace_replay import load_workloads, load_trace, record, replay_states, trace_items
    BinPacker, core = reference_packer()
    W = load_workloads()
    trace = load_trace("config3_seed1")
    seq = trace_items(trace)
    states = replay_states(trace, seq, positions)
    packer = BinPacker(W.TRAY3, num_orientations=24, interlocking_free=True)
    packer.pack_voxels([seq[0]])  # warm-up
    rows = []
    for pos in positions:
        item = seq[pos]
        core.gpu_tray_cleanup()  # see run_full
        t0 = time.perf_counter()
        res = packer.pack_voxels([item], initial_tray=states[pos])
        dt = time.perf_counter() - t0
        p = res.placements[0]
        want = trace["records"][pos]
        got = record(p.success, p.position, p.orientation_index, p.score)
        rows.append({"position": pos, "seconds": dt, "result": got, "oracle": want, "same": got == want})
    doc = {"rows": rows, "mean_seconds_per_item": float(np.mean([r["seconds"] for r in rows]))}
    Path(out).write_text(json.dumps(doc) + "\n")
    print(json.dumps(doc))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("mode", choices=["full", "sample"])
    ap.add_argument("--items", type=int, default=350)
    ap.add_argument("--positions", default="0,50,100,150,200,250,300")
    ap.add_argument("--out", default="ref_cuda.json")
    a = ap.parse_args()
    sys.path.insert(0, str(REPO))
    if a.mode == "full":
        run_full(a.items, a.out)
    else:
        run_sample([int(v) for v in a.positions.split(",")], a.out)


if __name__ == "__main__":
    main()
