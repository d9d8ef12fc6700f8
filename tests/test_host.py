"""Host-side logic: orientation order, packer argument checks, .vox layout, workloads."""
import numpy as np
import pytest

from oracle import psb_oracle as O
from psacking_b200 import BinPacker, workloads
from psacking_b200.rotations import apply_map, get_orientations, orientation_maps
from psacking_b200.vox import encode_vox


@pytest.mark.parametrize("n", [1, 4, 6, 24])
def test_orientations_match_reference_order(n):
    rng = np.random.default_rng(n)
    it = rng.integers(0, 4, (2, 3, 5))
    mine = get_orientations(it, n)
    ref = O.orientations(it, n)
    assert len(mine) == n
    assert all(np.array_equal(a, b) for a, b in zip(mine, ref))
    maps = orientation_maps(n)
    assert all(np.array_equal(apply_map(it, maps[k]), ref[k]) for k in range(n))


def test_24_orientations_distinct():
    it = np.arange(2 * 3 * 4).reshape(2, 3, 4)
    ors = get_orientations(it, 24)
    keys = {(o.shape, o.tobytes()) for o in ors}
    assert len(keys) == 24


def test_packer_validation():
    with pytest.raises(ValueError):
        BinPacker((10, 10))
    with pytest.raises(ValueError):
        BinPacker((10, -1, 10))
    with pytest.raises(ValueError):
        BinPacker((10, 10, 10), voxel_resolution=0)
    with pytest.raises(ValueError):
        BinPacker((10, 10, 10), num_orientations=5)
    p = BinPacker((10, 10, 10))
    with pytest.raises(ValueError, match="empty"):
        p.pack_voxels([])
    with pytest.raises(ValueError):
        p.pack_voxels([np.ones((2, 2))])
    assert "BinPacker(tray_size=(10, 10, 10)" in repr(p)


def test_vox_layout():
    g = np.zeros((2, 1, 3), np.int32)
    g[1, 0, 2] = 7
    b = encode_vox(g)
    assert np.frombuffer(b[:12], "<i4").tolist() == [2, 1, 3]
    body = np.frombuffer(b[12:12 + 6], np.uint8)
    # x from high to low, z from high to low: first byte is (1,0,2)
    assert body[0] == 123 + 7 % 5 and (body[1:] == 255).all()
    assert len(b) == 12 + 6 + 768


def test_vox_bytes_match_reference_save_vox():
    """encode_vox equals, byte for byte, the files the reference's own
    save_vox wrote for seeded grids (values 0, 8, above 255 and negative;
    tests/golden/ref_voxels.npz)."""
    import hashlib

    from tests import golden_vox
    cases = golden_vox.load_save_vox()
    assert len(cases) == 12
    for g, sha, n in cases:
        b = encode_vox(g)
        assert len(b) == n and hashlib.sha256(b).hexdigest() == sha


def test_workloads_deterministic_and_in_range():
    a = workloads.config1_items(3)
    b = workloads.config1_items(3)
    assert len(a) == 20 and all(np.array_equal(x, y) for x, y in zip(a, b))
    assert all(max(i.shape) <= 16 for i in a)
    c3 = workloads.config3_items(0, n=30)
    assert all(20 <= max(i.shape) <= 50 for i in c3)
    c2 = workloads.config2_items(0, n=10)
    assert all(max(i.shape) <= 40 for i in c2)


def test_positive_counts_match_numpy():
    """BinPacker's item volumes (cells > 0) are counted natively on the host
    cores; they must equal numpy's count for every item, with negative,
    zero and non-contiguous inputs among them."""
    from psacking_b200 import _core
    rng = np.random.default_rng(5)
    items = [rng.integers(-2, 4, tuple(rng.integers(1, 30, 3))).astype(np.int32) for _ in range(70)]
    items.append(np.zeros((3, 4, 5), np.int32))
    items.append(np.asfortranarray(rng.integers(0, 2, (9, 8, 7)).astype(np.int32)))
    want = [int(np.count_nonzero(a > 0)) for a in items]
    assert [int(v) for v in _core.positive_counts(items)] == want
    _, volumes, _, _, _ = BinPacker((40, 40, 40))._prepare(items, True, None)
    assert volumes == want


def test_rotation_matrices_match_reference_and_grids():
    """ROTATION_MATRICES_3x3 equals the reference's own list
    (tests/golden/ref_host.npz), and each matrix moves a voxel's centre
    (measured from the grid centre) to where get_24_orientations puts it."""
    from pathlib import Path

    from psacking_b200 import rotations as R
    want = np.load(Path(__file__).resolve().parent / "golden" / "ref_host.npz")["rotation_matrices_3x3"]
    assert len(R.ROTATION_MATRICES_3x3) == 24
    assert all(m.dtype == np.float64 and np.array_equal(m, w) for m, w in zip(R.ROTATION_MATRICES_3x3, want))
    g = np.zeros((2, 3, 5), np.int32)
    marks = [(0, 0, 0), (1, 2, 4), (1, 0, 3), (0, 2, 1)]
    for v, p in enumerate(marks, start=1):
        g[p] = v
    for o, og in enumerate(R.get_24_orientations(g)):
        m = R.get_rotation_matrix_3x3(o)
        assert np.allclose(m @ m.T, np.eye(3)) and np.isclose(np.linalg.det(m), 1.0)
        for v, p in enumerate(marks, start=1):
            src = np.asarray(p, float) - (np.asarray(g.shape) - 1) / 2
            dst = np.argwhere(og == v)[0] - (np.asarray(og.shape) - 1) / 2
            assert np.allclose(m @ src, dst), (o, v)
        m4 = R.get_rotation_matrix_4x4(o)
        assert np.array_equal(m4[:3, :3], m) and np.array_equal(m4[3], [0, 0, 0, 1]) and not m4[:3, 3].any()
    for bad in (-1, 24):
        with pytest.raises(IndexError):
            R.get_rotation_matrix_3x3(bad)


def test_pack_files_voxelizes_stl_then_packs(tmp_path, monkeypatch):
    """pack_files voxelizes every STL at the packer's voxel_resolution with
    voxelize_stl, in the order given, and hands the grids to pack_voxels
    (here the GPU voxelizer is replaced by its oracle and pack_voxels by a
    recorder: host logic only)."""
    from oracle import psb_voxel_oracle as V
    from psacking_b200 import voxelize as VZ
    from tests import meshes
    shapes = [meshes.box(), meshes.tetra(), meshes.icosphere(1)]
    paths = []
    for k, tris in enumerate(shapes):
        paths.append(tmp_path / f"m{k}.STL")
        VZ.write_stl(paths[-1], tris)
    monkeypatch.setattr(VZ, "voxelize_stl", lambda p, res: V.voxelize(VZ.read_stl(p), res))
    seen = {}

    def record(self, items, sort_by_volume=True, initial_tray=None):
        seen["items"], seen["sort"] = items, sort_by_volume
        return "packed"
    monkeypatch.setattr(BinPacker, "pack_voxels", record)
    bp = BinPacker((40, 40, 40), voxel_resolution=12)
    assert bp.pack_files([str(p) for p in paths], sort_by_volume=False) == "packed"
    assert seen["sort"] is False and len(seen["items"]) == 3
    for got, tris in zip(seen["items"], shapes):
        assert np.array_equal(got, V.voxelize(tris, 12))
    with pytest.raises(FileNotFoundError):
        bp.pack_files([tmp_path / "missing.stl"])
    (tmp_path / "x.obj").write_text("v 0 0 0\n")
    with pytest.raises(NotImplementedError):
        bp.pack_files([tmp_path / "x.obj"])


def test_pack_many_checkpoint_resumes_where_it_stopped(tmp_path, monkeypatch):
    """pack_many with a checkpoint: an interrupted call keeps the finished
    groups of trays, a resumed call packs only the rest, and the results
    equal an uninterrupted run; a checkpoint of other inputs is refused.
    _core.pack_many is replaced by the oracle's packing loop (host logic)."""
    from psacking_b200 import packer as PK
    calls = []

    def fake_pack_many(jobs, maps, interlock, concurrency):
        calls.append(len(jobs))
        outs = []
        for dims, items in jobs:
            tray, pl = O.pack_voxels(items, dims, 1, interlock, sort_by_volume=False)
            res = [((tuple(p["position"]) if p["success"] else (-1, -1, -1)), p["success"],
                    float(p["score"]) if p["success"] else 0.0, p["orientation_index"], 0, 0, 0.0) for p in pl]
            outs.append((tray, res))
        return outs
    monkeypatch.setattr(PK._core, "pack_many", fake_pack_many)
    rng = np.random.default_rng(5)
    trays = []
    for k in range(5):
        items = [np.ones(tuple(int(v) for v in rng.integers(2, 6, 3)), np.int32) for _ in range(4)]
        trays.append(((8, 9, 7), items))
    bp = BinPacker((8, 8, 8), num_orientations=1)
    full = bp.pack_many(trays, concurrency=2)
    ck = tmp_path / "run.npz"
    calls.clear()
    real = fake_pack_many

    def failing(jobs, *a):
        if len(calls) == 1:
            calls.append("fail")
            raise RuntimeError("interrupted")
        return real(jobs, *a)
    monkeypatch.setattr(PK._core, "pack_many", failing)
    with pytest.raises(RuntimeError, match="interrupted"):
        bp.pack_many(trays, concurrency=2, checkpoint=ck)
    with np.load(ck) as z:
        assert z["done"].tolist() == [0, 1]
    monkeypatch.setattr(PK._core, "pack_many", fake_pack_many)
    calls.clear()
    resumed = bp.pack_many(trays, concurrency=2, checkpoint=ck)
    assert calls == [2, 1]  # trays 2-4 only
    calls.clear()
    again = bp.pack_many(trays, concurrency=2, checkpoint=ck)
    assert calls == []
    for a, b, c in zip(full, resumed, again):
        assert np.array_equal(a.tray, b.tray) and np.array_equal(a.tray, c.tray)
        assert a.placements == b.placements == c.placements
        assert (a.num_placed, a.density) == (b.num_placed, b.density)
    with pytest.raises(ValueError, match="other trays"):
        bp.pack_many(trays[:4], concurrency=2, checkpoint=ck)
