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
