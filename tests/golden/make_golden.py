"""Generate tests/golden/ref_kats.npz from the reference's own test suite.

Run here (where the reference tree is mounted), never on the GPU box:

    python tests/golden/make_golden.py <reference checkout>

How it works: the reference's tests (tests/test_core.py, test_bindings.py,
test_distance_1d.py, test_distance_3d.py, test_distance_correctness.py,
test_flood_fill.py, test_orientations.py, and the whole-run suites
test_packer.py and test_interlocking.py, whose cage trays pin the
interlocking-free behaviour) import `spectral_packer`.  This script
puts a stand-in `spectral_packer` package on sys.path whose functions are the
CPU oracle (oracle/psb_oracle.py) and record every call.  It then runs those
reference tests with pytest.  A test passes only if the oracle's answers meet
the reference test's own expectations: the literal known-answer arrays, the
BFS / flood-fill CPU references written inside the test files, and the
behavioural assertions.  The calls made by passing tests, with their inputs
and the oracle outputs the reference accepted, become the golden fixture.
Arrays above 64k cells keep their input and a SHA-256 of the output.
"""
from __future__ import annotations

import hashlib
import json
import os
import pickle
import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
TEST_FILES = [
    "test_core.py", "test_bindings.py", "test_distance_1d.py", "test_distance_3d.py",
    "test_distance_correctness.py", "test_flood_fill.py", "test_orientations.py",
    "test_packer.py", "test_interlocking.py",
]
BIG = 65536

STUB = r'''
import os, pickle, sys, numpy as np
sys.path.insert(0, os.environ["PSB_REPO"])
from oracle import psb_oracle as O

_LOG = []
_CUR = {"test": None}

def _rec(name, args, out):
    _LOG.append((_CUR["test"], name, args, out))
    return out

def _arr(a):
    return np.array(a, copy=True)

def dft_conv3(a, b):
    return _rec("dft_conv3", (_arr(O.as_grid(a)), _arr(O.as_grid(b))), O.dft_conv3(a, b))
def dft_corr3(a, b):
    return _rec("dft_corr3", (_arr(O.as_grid(a)), _arr(O.as_grid(b))), O.dft_corr3(a, b))
def calculate_distance(g):
    return _rec("calculate_distance", (_arr(O.as_grid(g)),), O.calculate_distance(g))
def collision_grid(t, i):
    return _rec("collision_grid", (_arr(O.as_grid(t)), _arr(O.as_grid(i))), O.collision_grid(t, i))
def interlocking_free_positions(t, o):
    return _rec("interlocking_free_positions", (_arr(O.as_grid(t)), _arr(O.as_grid(o))),
                O.interlocking_free_positions(t, o))
def fft_search_placement(item, tray):
    r = O.fft_search_placement(item, tray)
    return _rec("fft_search_placement", (_arr(O.as_grid(item)), _arr(O.as_grid(tray))), r)
def fft_search_placement_with_cache(item, tray, tray_distance, generation=0):
    r = O.fft_search_placement_with_cache(item, tray, tray_distance, generation)
    return _rec("fft_search_placement_with_cache",
                (_arr(O.as_grid(item)), _arr(O.as_grid(tray)), _arr(O.as_grid(tray_distance))), r)
def fft_search_batch(orientations, tray, tray_distance, generation=0):
    pos, found, sc, _ = O.fft_search_batch(orientations, tray, tray_distance)
    r = (pos, found, sc)
    return _rec("fft_search_batch",
                ([_arr(O.as_grid(o)) for o in orientations], _arr(O.as_grid(tray)),
                 _arr(O.as_grid(tray_distance))), r)
def fft_search_batch_interlocking_free(orientations, tray, tray_distance, generation=0):
    r = O.fft_search_batch(orientations, tray, tray_distance, interlock=True)
    return _rec("fft_search_batch_interlocking_free",
                ([_arr(O.as_grid(o)) for o in orientations], _arr(O.as_grid(tray)),
                 _arr(O.as_grid(tray_distance))), r)
def place_in_tray(item, tray, position, item_id=1):
    r = O.place_in_tray(item, tray, position, item_id)
    return _rec("place_in_tray", (_arr(O.as_grid(item)), _arr(O.as_grid(tray)), tuple(position), item_id), r)
def make_tight(g):
    return O.make_tight(g)
def get_bounds(g):
    return O.bounds(O.as_grid(g))

rotate_90_x, rotate_90_y, rotate_90_z = O._rx, O._ry, O._rz
def get_orientations(grid, num_orientations=1):
    return O.orientations(grid, num_orientations)
def get_24_orientations(grid):
    return O.orientations(grid, 24)

class PlacementInfo:
    def __init__(self, d):
        self.item_index = d["item_index"]
        self.position = d["position"]
        self.score = d["score"]
        self.success = d["success"]
        self.volume = d["volume"]
        self.orientation_index = d["orientation_index"]

class PackingResult:
    def __init__(self, tray, placements):
        self.tray = tray
        self.placements = placements
        self.num_placed = sum(1 for p in placements if p.success)
        self.num_failed = len(placements) - self.num_placed
        self.density = O.density(tray)
        self.total_volume = int((tray > 0).sum())
        idx = np.argwhere(tray > 0)
        self.bounding_box = (tuple(int(v) for v in idx.min(axis=0)), tuple(int(v) for v in idx.max(axis=0))) \
            if len(idx) else None
    def get_item_mask(self, item_id):
        return self.tray == item_id
    def summary(self):
        return ("Packing Result Summary\n" f"Items placed: {self.num_placed}\n"
                f"Packing density: {self.density:.1%}\n")

class BinPacker:
    def __init__(self, tray_size, voxel_resolution=128, height_penalty=1e8,
                 num_orientations=1, interlocking_free=False):
        if len(tray_size) != 3:
            raise ValueError("tray_size must be a 3-tuple")
        if any(s <= 0 for s in tray_size):
            raise ValueError("tray_size dimensions must be positive")
        if voxel_resolution <= 0:
            raise ValueError("voxel_resolution must be positive")
        if num_orientations not in (1, 4, 6, 24):
            raise ValueError("num_orientations must be 1, 4, 6, or 24")
        self.tray_size = tuple(tray_size)
        self.voxel_resolution = voxel_resolution
        self.height_penalty = height_penalty
        self.num_orientations = num_orientations
        self.interlocking_free = interlocking_free
    def __repr__(self):
        return f"BinPacker(tray_size={self.tray_size}, voxel_resolution={self.voxel_resolution})"
    def pack_voxels(self, items, sort_by_volume=True, initial_tray=None):
        if len(items) == 0:
            raise ValueError("items list cannot be empty")
        tray, pl = O.pack_voxels(items, self.tray_size, self.num_orientations,
                                 self.interlocking_free, sort_by_volume, initial_tray)
        _rec("pack_voxels", ([np.array(i) for i in items], self.tray_size, self.num_orientations,
                             self.interlocking_free, sort_by_volume,
                             None if initial_tray is None else _arr(O.as_grid(initial_tray))),
             (tray, [(p["position"], p["success"], p["orientation_index"], p["score"]) for p in pl]))
        return PackingResult(tray, [PlacementInfo(p) for p in pl])
    def pack_single(self, item, tray=None):
        if tray is None:
            tray = np.zeros(self.tray_size, dtype=np.int32)
        pos, found, sc = fft_search_placement(np.asarray(item).astype(np.int32), tray)
        return (tuple(pos), True, sc) if found else (None, False, 0.0)

def _dump(path):
    with open(path, "wb") as f:
        pickle.dump(_LOG, f)
'''

PLUGIN = r'''
import os, spectral_packer as sp
_OUT = {}
def pytest_runtest_setup(item):
    sp._CUR["test"] = item.nodeid
def pytest_runtest_logreport(report):
    if report.when == "call":
        _OUT[report.nodeid] = report.outcome
def pytest_sessionfinish(session, exitstatus):
    import json
    sp._dump(os.environ["PSB_LOG"])
    with open(os.environ["PSB_OUTCOMES"], "w") as f:
        json.dump(_OUT, f)
'''


def _pack(obj):
    """Pickle-free encoding: nested tuples/lists/arrays -> JSON + arrays."""
    arrays = []

    def enc(x):
        if isinstance(x, np.ndarray):
            if x.size > BIG:
                pass
            arrays.append(np.ascontiguousarray(x))
            return {"__a__": len(arrays) - 1}
        if isinstance(x, (list, tuple)):
            return {"__t__": isinstance(x, tuple), "v": [enc(v) for v in x]}
        if isinstance(x, (np.integer,)):
            return int(x)
        if isinstance(x, (np.floating,)):
            return float(x)
        if isinstance(x, (np.bool_,)):
            return bool(x)
        return x
    return enc(obj), arrays


def main(ref_root):
    ref_tests = Path(ref_root) / "tests"
    if not ref_tests.is_dir():
        raise SystemExit(f"{ref_tests} is not a directory: pass the reference checkout")
    work = Path(tempfile.mkdtemp(prefix="psb_golden_"))
    try:
        (work / "spectral_packer").mkdir()
        (work / "spectral_packer" / "__init__.py").write_text(STUB)
        (work / "psb_plugin.py").write_text(PLUGIN)
        tdir = work / "tests"
        tdir.mkdir()
        for f in ["conftest.py", "__init__.py"] + TEST_FILES:
            if (ref_tests / f).exists():
                shutil.copy(ref_tests / f, tdir / f)
        env = dict(os.environ, PSB_REPO=str(REPO), PSB_LOG=str(work / "log.pkl"),
                   PSB_OUTCOMES=str(work / "outcomes.json"),
                   PYTHONPATH=str(work), PYTHONDONTWRITEBYTECODE="1", MPLBACKEND="Agg")
        cmd = [sys.executable, "-m", "pytest", "-q", "-p", "psb_plugin", "-p", "no:cacheprovider",
               "--rootdir", str(work), "-k", "not benchmark and not Benchmark",
               *[str(tdir / f) for f in TEST_FILES]]
        r = subprocess.run(cmd, cwd=work, env=env, capture_output=True, text=True)
        print(r.stdout[-3000:])
        print(r.stderr[-2000:])
        outcomes = json.loads((work / "outcomes.json").read_text())
        with open(work / "log.pkl", "rb") as f:
            log = pickle.load(f)
    finally:
        shutil.rmtree(work, ignore_errors=True)

    records, arrays = [], []
    for test, name, args, out in log:
        if outcomes.get(test) != "passed":
            continue
        rec_args, a1 = _pack(args)
        base = len(arrays)
        arrays.extend(a1)

        def shift(x):
            if isinstance(x, dict) and "__a__" in x:
                return {"__a__": x["__a__"] + base}
            if isinstance(x, dict) and "v" in x:
                return {"__t__": x["__t__"], "v": [shift(v) for v in x["v"]]}
            return x
        rec_args = shift(rec_args)
        if isinstance(out, np.ndarray) and out.size > BIG:
            rec_out = {"__sha__": hashlib.sha256(np.ascontiguousarray(out, dtype=np.int32).tobytes()).hexdigest(),
                       "shape": list(out.shape)}
        else:
            rec_out, a2 = _pack(out)
            base2 = len(arrays)
            arrays.extend(a2)
            base = base2
            rec_out = shift(rec_out)
        records.append({"test": test.split("tests/")[-1], "fn": name, "args": rec_args, "out": rec_out})
    np.savez_compressed(HERE / "ref_kats.npz", index=np.array(json.dumps(records)),
                        **{f"a{i}": a for i, a in enumerate(arrays)})
    n_pass = sum(1 for v in outcomes.values() if v == "passed")
    print(f"{len(records)} golden calls from {n_pass}/{len(outcomes)} passing reference tests")
    fails = [k for k, v in outcomes.items() if v != "passed"]
    (HERE / "ref_kats_outcomes.json").write_text(json.dumps(
        {"passed": n_pass, "total": len(outcomes), "not_passed": fails}, indent=1))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: python tests/golden/make_golden.py <reference checkout>")
    main(sys.argv[1])
