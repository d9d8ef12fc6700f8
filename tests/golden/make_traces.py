"""Generate the golden packing traces in tests/golden/traces/ with the oracle.

    python tests/golden/make_traces.py [--only NAME ...] [--jobs N]

Each trace is one whole greedy packing run of a seeded workload, computed by
the CPU oracle (oracle/psb_oracle.py, the reference's algorithm in exact
arithmetic; BinPacker.pack_voxels, spectral_packer/packer.py:366-544):

  config1_seed0 .. config1_seed9  64^3 tray, 20 box-union items, 1 orientation
                                  (fft_search_placement, packing.cpp:590-642)
  config2_seed0                   128^3 tray, 100 items, 24 orientations
                                  (fft_search_placement_with_cache, fft3.cu:1506-1521)
  config3_seed1                   240x123x100 tray, 350 items, 24 orientations,
                                  interlocking-free (fft3.cu:1589-1632); the
                                  item stream the benchmark packs

A trace records, per item in search order (descending volume, the order
np.argsort(volumes)[::-1] gives), (found, x, y, z, orientation, score), plus
the SHA-256 of the final int32 tray, its density and the placed count.  The
GPU tests and bench.py compare the device-resident loop with these records
position by position.  The workloads module is loaded by path, so this script
needs neither the built extension nor a GPU.  The config-3 trace takes about
half an hour on 8 cores.
"""
from __future__ import annotations

import argparse
import hashlib
import importlib.util
import json
import sys
import time
from concurrent.futures import ProcessPoolExecutor
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
OUT = HERE / "traces"
sys.path.insert(0, str(REPO))


def load_workloads():
    spec = importlib.util.spec_from_file_location("psb_workloads", REPO / "psacking_b200" / "workloads.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def traces():
    W = load_workloads()
    out = {f"config1_seed{s}": dict(gen="config1_items", seed=s, n=20, tray=W.TRAY1, n_orient=1, interlock=False)
           for s in range(10)}
    out["config2_seed0"] = dict(gen="config2_items", seed=0, n=100, tray=W.TRAY2, n_orient=24, interlock=False)
    out["config3_seed1"] = dict(gen="config3_items", seed=1, n=350, tray=W.TRAY3, n_orient=24, interlock=True)
    return out


def search_order(items):
    vols = [int(np.sum(np.asarray(i) > 0)) for i in items]
    return [int(i) for i in np.argsort(vols)[::-1]]


def make(name: str) -> str:
    from oracle import psb_oracle as O
    W = load_workloads()
    spec = traces()[name]
    items = getattr(W, spec["gen"])(spec["seed"], n=spec["n"])
    order = search_order(items)
    t0 = time.time()

    def progress(n, p):
        if n % 25 == 0:
            print(f"{name}: {n}/{len(items)} items, {time.time() - t0:.0f} s", flush=True)

    tray, pl = O.pack_voxels(items, spec["tray"], spec["n_orient"], spec["interlock"], True, fast=True,
                             progress=progress)
    by_index = {p["item_index"]: p for p in pl}
    records = []
    for i in order:
        p = by_index[i]
        if p["success"]:
            records.append([1, *[int(v) for v in p["position"]], int(p["orientation_index"]), float(p["score"])])
        else:
            records.append([0, -1, -1, -1, 0, 0.0])
    doc = {"name": name, "generator": spec["gen"], "seed": spec["seed"], "n_items": spec["n"],
           "tray": list(spec["tray"]), "num_orientations": spec["n_orient"], "interlocking_free": spec["interlock"],
           "order": order, "records": records,
           "tray_sha256": hashlib.sha256(np.ascontiguousarray(tray, dtype=np.int32).tobytes()).hexdigest(),
           "num_placed": int(sum(r[0] for r in records)), "density": O.density(tray),
           "oracle_seconds": round(time.time() - t0, 1)}
    OUT.mkdir(exist_ok=True)
    (OUT / f"{name}.json").write_text(json.dumps(doc, separators=(",", ":")) + "\n")
    return f"{name}: {doc['num_placed']}/{spec['n']} placed, density {doc['density']:.4f}, {doc['oracle_seconds']} s"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", nargs="*", help="trace names (default: all)")
    ap.add_argument("--jobs", type=int, default=1, help="traces generated at once (separate processes)")
    a = ap.parse_args()
    names = a.only or list(traces())
    if a.jobs <= 1:
        for n in names:
            print(make(n), flush=True)
        return
    import multiprocessing as mp
    with ProcessPoolExecutor(a.jobs, mp_context=mp.get_context("spawn")) as ex:
        for msg in ex.map(make, names):
            print(msg, flush=True)


if __name__ == "__main__":
    main()
