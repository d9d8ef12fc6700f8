"""The oracle's host functions against the reference's own module
(tests/golden/ref_host.npz, recorded by tests/golden/make_host_golden.py
from the reference built from its sources): place_in_tray on items partly
outside the tray, negative positions and values, and overlaps (same error
and the same first overlapping cell); get_bounds and make_tight on sparse,
single-voxel, full and empty grids."""
from pathlib import Path

import numpy as np
import pytest

from oracle import psb_oracle as O

Z = np.load(Path(__file__).resolve().parent / "golden" / "ref_host.npz")


@pytest.mark.parametrize("k", range(int(Z["place_count"])))
def test_place_in_tray_matches_reference(k):
    item, tray = Z[f"place/{k}/item"], Z[f"place/{k}/tray"]
    pos, val = tuple(int(v) for v in Z[f"place/{k}/pos"]), int(Z[f"place/{k}/val"])
    if f"place/{k}/error" in Z.files:
        with pytest.raises(RuntimeError) as e:
            O.place_in_tray(item, tray, pos, val)
        assert str(e.value) == str(Z[f"place/{k}/error"])
        return
    out = O.place_in_tray(item, tray, pos, val)
    assert out.dtype == np.int32 and np.array_equal(out, Z[f"place/{k}/out"])


def test_place_fixture_covers_both_outcomes():
    n = int(Z["place_count"])
    errors = sum(f"place/{k}/error" in Z.files for k in range(n))
    assert 0 < errors < n


@pytest.mark.parametrize("k", range(int(Z["grid_count"])))
def test_bounds_and_tight_match_reference(k):
    g = Z[f"grid/{k}/in"]
    lo, hi = O.bounds(g)
    assert [list(lo), list(hi)] == Z[f"grid/{k}/bounds"].tolist()
    if f"grid/{k}/tight_error" in Z.files:
        with pytest.raises(ValueError):
            O.make_tight(g)
        return
    t = O.make_tight(g)
    want = Z[f"grid/{k}/tight"]
    assert t.shape == want.shape and np.array_equal(t, want)


@pytest.mark.parametrize("k", range(int(Z["stats_count"])))
def test_packing_stats_and_summary_match_reference(k):
    """BinPacker's density / volume / bounding box, from the tray on the
    host (_calculate_stats) and from the device's counts (_stats_from_counts,
    fed here with numpy's), PackingResult.summary() and BinPacker's repr equal
    the reference's on the same trays (packer.py:145-162, 582-608)."""
    from psacking_b200 import BinPacker, PackingResult
    tray = Z[f"stats/{k}/tray"]
    res, n_or, placed, failed = (int(v) for v in Z[f"stats/{k}/args"])
    bp = BinPacker(tray.shape, voxel_resolution=res, num_orientations=n_or)
    bbox = Z[f"stats/{k}/bbox"].tolist()
    want = (float(Z[f"stats/{k}/density"]), int(Z[f"stats/{k}/total"]),
            None if bbox[0][0] < 0 else (tuple(bbox[0]), tuple(bbox[1])))
    assert bp._calculate_stats(tray) == want
    occ = np.argwhere(tray > 0)
    lo, hi = (occ.min(axis=0), occ.max(axis=0)) if len(occ) else ((0, 0, 0), (-1, -1, -1))
    assert BinPacker._stats_from_counts(len(occ), lo, hi) == want
    r = PackingResult(tray=tray, num_placed=placed, num_failed=failed, density=want[0], total_volume=want[1],
                      bounding_box=want[2])
    assert r.summary() == str(Z[f"stats/{k}/summary"])
    assert repr(bp) == str(Z[f"stats/{k}/repr"])
