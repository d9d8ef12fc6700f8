"""The CPU oracle reproduces every golden call the reference's own tests accepted."""
import numpy as np
import pytest

from oracle import psb_oracle as O
from tests.golden_io import load_records, same_output

RECORDS = load_records()
FUNCS = {
    "dft_conv3": lambda a: O.dft_conv3(*a),
    "dft_corr3": lambda a: O.dft_corr3(*a),
    "calculate_distance": lambda a: O.calculate_distance(*a),
    "collision_grid": lambda a: O.collision_grid(*a),
    "interlocking_free_positions": lambda a: O.interlocking_free_positions(*a),
    "fft_search_placement": lambda a: O.fft_search_placement(*a),
    "fft_search_placement_with_cache": lambda a: O.fft_search_placement_with_cache(*a),
    "fft_search_batch": lambda a: O.fft_search_batch(*a)[:3],
    "place_in_tray": lambda a: O.place_in_tray(*a),
    "pack_voxels": lambda a: _pack(a),
}


def _pack(a):
    items, tray_size, n_orient, interlock, sort = a[:5]
    initial = a[5] if len(a) > 5 else None
    tray, pl = O.pack_voxels(items, tuple(tray_size), n_orient, interlock, sort, initial_tray=initial)
    return (tray, [(None if p["position"] is None else tuple(p["position"]), p["success"],
                    p["orientation_index"], p["score"]) for p in pl])


def test_golden_fixture_nonempty():
    fns = {r["fn"] for r in RECORDS}
    assert {"dft_conv3", "dft_corr3", "calculate_distance", "interlocking_free_positions",
            "fft_search_placement", "place_in_tray"} <= fns
    assert len(RECORDS) > 100


@pytest.mark.parametrize("i", [i for i, r in enumerate(RECORDS) if r["fn"] in FUNCS])
def test_oracle_matches_golden(i):
    r = RECORDS[i]
    got = FUNCS[r["fn"]](r["args"])
    assert same_output(got, r["out"]), (r["test"], r["fn"])


def test_literal_kats():
    # spot checks straight from the reference's known-answer tests (tests/test_core.py:17-152)
    a = np.array([[[1, 1, 1]]], np.int32)
    b = np.array([[[1, 2, 3]]], np.int32)
    assert O.dft_conv3(a, b).tolist() == [[[1, 3, 6]]]
    assert O.dft_corr3(a, b).tolist() == [[[6, 3, 1]]]
    t = np.zeros((3, 1, 4), np.int32)
    t[1, 0, 1] = 1
    assert O.calculate_distance(t)[:, 0, :].tolist() == [[2, 1, 2, 3], [1, 0, 1, 2], [2, 1, 2, 3]]
