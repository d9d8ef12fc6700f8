"""Whole packing runs on the GPU against the oracle's golden traces.

Every trace in tests/golden/traces is one greedy run of a seeded workload
computed by the oracle (tests/golden/make_traces.py): config 1 seeds 0-9
(64^3, 20 items, 1 orientation), config 2 seed 0 (128^3, 100 items, 24
orientations) and config 3 seed 1 (240x123x100, 350 items, 24 orientations,
interlocking-free: the benchmark's own stream, where the candidate
pre-filter, the direct decisions and nz = 100 -- four 32-bit words, the last
one partial -- all take part).  The device-resident loop must reproduce every
item's (found, position, orientation, score) bit for bit and the final tray's
SHA-256, with the engine's defaults and with the pre-filter off; the
reference's call pattern (engine="calls") must too.
"""
import hashlib
from pathlib import Path

import numpy as np
import pytest

from oracle.trace_replay import load_trace, trace_items

pytestmark = pytest.mark.gpu

TRACES = sorted(p.stem for p in (Path(__file__).resolve().parent / "golden" / "traces").glob("*.json"))


def _records(res):
    return [[1, *p.position, p.orientation_index, p.score] if p.success else [0, -1, -1, -1, 0, 0.0]
            for p in res.placements]


def _run(name, engine="native"):
    from psacking_b200 import BinPacker
    tr = load_trace(name)
    seq = trace_items(tr)
    res = BinPacker(tuple(tr["tray"]), num_orientations=tr["num_orientations"],
                    interlocking_free=tr["interlocking_free"], engine=engine).pack_voxels(seq, sort_by_volume=False)
    return tr, res


def _check(tr, res):
    got = _records(res)
    bad = [i for i, (a, b) in enumerate(zip(got, tr["records"])) if a != b]
    assert not bad, (tr["name"], bad[0], got[bad[0]], tr["records"][bad[0]])
    assert hashlib.sha256(np.ascontiguousarray(res.tray, np.int32).tobytes()).hexdigest() == tr["tray_sha256"]
    assert res.num_placed == tr["num_placed"]
    assert res.density == tr["density"]
    # the statistics counted on the device equal the host computation
    from psacking_b200 import BinPacker
    want = BinPacker(tuple(tr["tray"]))._calculate_stats(res.tray)
    assert (res.density, res.total_volume, res.bounding_box) == want


@pytest.mark.parametrize("name", TRACES)
def test_native_loop_matches_trace(gpu_core, name):
    tr, res = _run(name)
    _check(tr, res)


@pytest.mark.parametrize("name", ["config2_seed0", "config3_seed1"])
def test_native_loop_matches_trace_filter_off(gpu_core, name):
    gpu_core.set_cand_filter(False)
    try:
        tr, res = _run(name)
    finally:
        gpu_core.set_cand_filter(True)
    _check(tr, res)


@pytest.mark.parametrize("name", ["config3_seed1"])
def test_native_loop_matches_trace_every_sample(gpu_core, name):
    """The pre-filter with every sample tested and direct decisions up to a
    larger limit (16384 candidates): more orientations decided without
    transforms."""
    gpu_core.set_filter_cut(0)
    gpu_core.set_direct_max(16384)
    try:
        tr, res = _run(name)
    finally:
        gpu_core.set_filter_cut(50)
        gpu_core.set_direct_max(4096)
    _check(tr, res)


@pytest.mark.parametrize("late", [1024, 1 << 16])
@pytest.mark.parametrize("name", ["config2_seed0", "config3_seed1"])
def test_native_loop_matches_trace_late_direct(gpu_core, name, late):
    """Orientations left with few ok cells after the collision pass take
    exact proximity sums instead of the proximity transforms (off by
    default): up to 1024 ok cells, or practically all (2^16 cells)."""
    gpu_core.set_late_direct_max(late)
    try:
        tr, res = _run(name)
    finally:
        gpu_core.set_late_direct_max(0)
    _check(tr, res)


@pytest.mark.parametrize("name", ["config1_seed0", "config1_seed9", "config2_seed0", "config3_seed1"])
def test_call_pattern_matches_trace(gpu_core, name):
    tr, res = _run(name, engine="calls")
    _check(tr, res)
