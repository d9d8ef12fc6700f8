"""Tray states of a golden packing trace -- TEST INFRASTRUCTURE ONLY.

A trace (tests/golden/traces/*.json, written by tests/golden/make_traces.py)
records one oracle packing run item by item.  replay_states rebuilds the tray
as it was before any listed search position: placed items are written with
ids 1, 2, ... in placement order (item_id = id_offset + num_placed + 1,
spectral_packer/packer.py:508-509), each in its recorded orientation
(get_24_orientations, spectral_packer/rotations.py:159-219) at its recorded
origin.  The benchmark's CPU sample and the reference's GPU sample search the
items of the stream against these states.
"""
from __future__ import annotations

import importlib.util
import json
from pathlib import Path

import numpy as np

from .psb_oracle import orientations

REPO = Path(__file__).resolve().parent.parent
TRACES = REPO / "tests" / "golden" / "traces"


def load_workloads():
    """psacking_b200/workloads.py loaded by path: it needs only numpy, and
    importing the package would load the engine's shared libraries."""
    spec = importlib.util.spec_from_file_location("psb_workloads", REPO / "psacking_b200" / "workloads.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def load_trace(name: str) -> dict:
    return json.loads((TRACES / f"{name}.json").read_text())


def trace_items(trace: dict):
    """The trace's items in search order (checked against the recorded order)."""
    W = load_workloads()
    items = getattr(W, trace["generator"])(trace["seed"], n=trace["n_items"])
    vols = [int(np.sum(np.asarray(i) > 0)) for i in items]
    order = [int(i) for i in np.argsort(vols)[::-1]]
    if order != trace["order"]:
        raise AssertionError(f"{trace['name']}: item order differs from the trace")
    return [np.ascontiguousarray(items[i], dtype=np.int32) for i in order]


def oriented(item, o: int, n_orient: int) -> np.ndarray:
    return np.ascontiguousarray(orientations(np.asarray(item, np.int32), n_orient)[o])


def replay_states(trace: dict, seq, positions):
    """{position: tray before the item at that search position}."""
    want = sorted(set(int(p) for p in positions))
    tray = np.zeros(tuple(trace["tray"]), np.int32)
    states, placed, p = {}, 0, 0
    recs = trace["records"]
    for pos in want:
        while p < pos:
            f, x, y, z, o, _ = recs[p]
            if f:
                placed += 1
                it = oriented(seq[p], int(o), trace["num_orientations"])
                sub = tray[x:x + it.shape[0], y:y + it.shape[1], z:z + it.shape[2]]
                if np.any((sub > 0) & (it > 0)):
                    raise AssertionError(f"trace record {p} overlaps the replayed tray")
                sub[it > 0] = placed
            p += 1
        states[pos] = tray.copy()
    return states


def record(found, pos, orient, score):
    """A result in the trace's record form [found, x, y, z, orientation, score]."""
    if not found:
        return [0, -1, -1, -1, 0, 0.0]
    return [1, int(pos[0]), int(pos[1]), int(pos[2]), int(orient), float(score)]
