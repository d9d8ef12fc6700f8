"""Device-side limits and host-side failures end in an error status, never in
a spin or a leak.

* The flood fill's union-find gives up after a bounded number of steps
  (psb_set_uf_limit).  With the bound set to 1 on trays whose free space forms
  long chains of z-runs, the searches and the packing loop return
  PSB_ERR_LIMIT (RuntimeError in the drop-in module): the kernels returned.
  With the default bound restored, the same calls give the oracle's answers,
  so the context stayed usable.
* Device allocation failures, injected at every allocation of a tray's
  creation and of a packing run, return PSB_ERR_CUDA and free everything the
  failed call allocated (the engine's live-allocation count returns to where
  it was).
"""
import ctypes
from pathlib import Path

import numpy as np
import pytest

from oracle import psb_oracle as O

pytestmark = pytest.mark.gpu

LIB = Path(__file__).resolve().parent.parent / "psacking_b200" / "libpsb200.so"
PSB_ERR_CUDA, PSB_ERR_LIMIT = 2, 5


def serpentine_tray(n=33, nz=3):
    """Walls everywhere except a one-cell-high corridor at z = 1 that snakes
    through the x-y plane and opens on the face x = 0: every free cell is
    reachable, through one long chain of single-cell runs."""
    tray = np.full((n, n, nz), 2, np.int32)
    for y in range(1, n - 1, 2):
        tray[1:n - 1, y, 1] = 0
        if y + 2 < n - 1:
            link_x = n - 2 if (y // 2) % 2 == 0 else 1
            tray[link_x, y + 1, 1] = 0
    tray[0, 1, 1] = 0
    return tray


def random_tray(seed, shape=(48, 40, 36), fill=0.3):
    rng = np.random.default_rng(seed)
    return (rng.random(shape) < fill).astype(np.int32) * 2


def boxes_tray(seed, shape=(40, 40, 24), n_boxes=8):
    """Mostly open space with a few solid boxes: one large free region made
    of many z-runs, so the union-find merges long chains for every item."""
    rng = np.random.default_rng(seed)
    tray = np.zeros(shape, np.int32)
    for _ in range(n_boxes):
        e = [int(rng.integers(3, s // 3)) for s in shape]
        o = [int(rng.integers(0, s - ee)) for s, ee in zip(shape, e)]
        tray[o[0]:o[0] + e[0], o[1]:o[1] + e[1], o[2]:o[2] + e[2]] = 2
    return tray


@pytest.fixture
def uf_limit(gpu_core):
    yield gpu_core.set_uf_limit
    gpu_core.set_uf_limit(0)


def test_flood_fill_limit_returns_error_then_recovers(gpu_core, uf_limit):
    item = np.ones((1, 1, 1), np.int32)
    for tray in (serpentine_tray(), random_tray(1)):
        want = O.interlocking_free_positions(tray, item)
        uf_limit(1)
        with pytest.raises(RuntimeError, match="iteration limit"):
            gpu_core.interlocking_free_positions(tray, item)
        uf_limit(0)
        np.testing.assert_array_equal(gpu_core.interlocking_free_positions(tray, item), want)


def test_search_limit_returns_error_then_recovers(gpu_core, uf_limit):
    """Every orientation's own result (per_orientation=True) runs the flood
    fill for all of them; the drop-in batch search runs it only when its
    winner has no straight free run to a seed face, which here it has."""
    tray = boxes_tray(2)
    phi = O.calculate_distance(tray)
    ors = [np.ones((2, 1, 1), np.int32), np.ones((1, 2, 2), np.int32)]
    flags = 1 | 0x10   # PSB_MODE_BLOCK | PSB_FLAG_INTERLOCK
    want = O.fft_search_batch(ors, tray, phi, interlock=True)
    gpu_core.gpu_tray_init(tray, phi)
    uf_limit(1)
    with pytest.raises(RuntimeError, match="iteration limit"):
        gpu_core.search_detail(ors, flags, per_orientation=True)
    uf_limit(0)
    d = gpu_core.search_detail(ors, flags, per_orientation=True)
    pos, found, score, bo = d["best"]
    assert (tuple(pos), found, score, bo) == (tuple(want[0]), want[1], want[2], want[3])
    gpu_core.gpu_tray_cleanup()


def test_packing_loop_limit_returns_error_then_recovers(gpu_core, uf_limit):
    """A 64^3 tray (specialised FFT lengths): the loop's search runs the flood
    fill for every item (other lengths take the lazy interlocking flow, which
    skips it when the winner has a straight free run to a seed face)."""
    from psacking_b200 import BinPacker, workloads
    items = workloads.config1_items(2)[:5]
    tray = boxes_tray(3, shape=(64, 64, 64))
    packer = BinPacker(tray.shape, num_orientations=4, interlocking_free=True)
    uf_limit(1)
    with pytest.raises(RuntimeError, match="iteration limit"):
        packer.pack_voxels(items, initial_tray=tray)
    uf_limit(0)
    got = packer.pack_voxels(items, initial_tray=tray)
    want_tray, want = O.pack_voxels(items, tray.shape, 4, True, initial_tray=tray)
    np.testing.assert_array_equal(got.tray, want_tray)
    assert [(p.success, p.position, p.orientation_index) for p in got.placements] == \
           [(w["success"], w["position"], w["orientation_index"]) for w in want]


class _Abi:
    def __init__(self):
        self.lib = lib = ctypes.CDLL(str(LIB))
        P, I = ctypes.c_void_p, ctypes.c_int
        lib.psb_last_error.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
        lib.psb_debug_fail_alloc.argtypes = [I]
        lib.psb_debug_live_allocs.argtypes = [P]
        lib.psb_tray_create.argtypes = [I, I, I, P]
        lib.psb_tray_destroy.argtypes = [P]
        lib.psb_tray_set.argtypes = [P, P, P]
        lib.psb_pack.argtypes = [P, P, P, I, P, I, I, ctypes.c_int32, P, P]

    def err(self):
        buf = ctypes.create_string_buffer(1024)
        self.lib.psb_last_error(buf, 1024)
        return buf.value.decode()

    def live(self):
        n = ctypes.c_longlong(-1)
        assert self.lib.psb_debug_live_allocs(ctypes.byref(n)) == 0
        return n.value


def test_injected_allocation_failures_are_clean():
    abi = _Abi()
    lib = abi.lib
    base = abi.live()
    # every allocation of a tray's creation, one at a time
    failures = 0
    for k in range(1, 64):
        lib.psb_debug_fail_alloc(k)
        t = ctypes.c_void_p()
        st = lib.psb_tray_create(40, 36, 30, ctypes.byref(t))
        lib.psb_debug_fail_alloc(0)
        if st == 0:
            assert lib.psb_tray_destroy(t) == 0
            break
        assert st == PSB_ERR_CUDA and "injected" in abi.err(), (k, st, abi.err())
        assert not t.value
        assert abi.live() == base, k
        failures += 1
    assert failures >= 10   # the tray allocates its grids, spectra and work buffers
    # every allocation of a packing run (staging, slots, loop buffers)
    from psacking_b200 import workloads
    from psacking_b200.rotations import orientation_maps
    items = [np.ascontiguousarray(i) for i in workloads.config1_items(5)[:4]]
    ptrs = (ctypes.POINTER(ctypes.c_int32) * len(items))(
        *[i.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)) for i in items])
    dims = np.array([i.shape for i in items], np.int32).ravel()
    maps = np.ascontiguousarray(orientation_maps(4), np.int32)
    tray0 = np.zeros((40, 36, 30), np.int32)

    class Res(ctypes.Structure):
        _fields_ = [("x", ctypes.c_int32), ("y", ctypes.c_int32), ("z", ctypes.c_int32),
                    ("found", ctypes.c_int32), ("score", ctypes.c_double), ("orientation", ctypes.c_int32),
                    ("diag", ctypes.c_uint32), ("n_candidates", ctypes.c_int32), ("err_ratio", ctypes.c_float)]

    def pack(k):
        t = ctypes.c_void_p()
        assert lib.psb_tray_create(40, 36, 30, ctypes.byref(t)) == 0, abi.err()
        assert lib.psb_tray_set(t, tray0.ctypes.data, None) == 0, abi.err()
        res = (Res * len(items))()
        out = np.zeros_like(tray0)
        lib.psb_debug_fail_alloc(k)
        st = lib.psb_pack(t, ptrs, dims.ctypes.data, len(items), maps.ctypes.data, 4, 1, 0, res, out.ctypes.data)
        lib.psb_debug_fail_alloc(0)
        msg = abi.err()
        assert lib.psb_tray_destroy(t) == 0
        return st, msg, res, out

    failures = 0
    for k in range(1, 128):
        st, msg, res, out = pack(k)
        assert abi.live() == base, k
        if st == 0:
            break
        assert st == PSB_ERR_CUDA and "injected" in msg, (k, st, msg)
        failures += 1
    assert failures >= 3
    want_tray, want = O.pack_voxels(items, tray0.shape, 4, True, sort_by_volume=False)
    np.testing.assert_array_equal(out, want_tray)


def test_injected_allocation_failures_streamed_staging_are_clean():
    """psb_pack with 64 items or more stages them in two parts, the second
    one uploaded (and its item columns computed) while the first part is
    searched: an allocation failure anywhere, including mid-run, returns
    PSB_ERR_CUDA, and destroying the tray frees everything."""
    abi = _Abi()
    lib = abi.lib
    base = abi.live()
    from psacking_b200 import workloads
    from psacking_b200.rotations import orientation_maps
    items = [np.ascontiguousarray(i) for s in range(4) for i in workloads.config1_items(s)][:70]
    ptrs = (ctypes.POINTER(ctypes.c_int32) * len(items))(
        *[i.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)) for i in items])
    dims = np.array([i.shape for i in items], np.int32).ravel()
    maps = np.ascontiguousarray(orientation_maps(4), np.int32)
    shape = (64, 64, 40)
    tray0 = np.zeros(shape, np.int32)

    class Res(ctypes.Structure):
        _fields_ = [("x", ctypes.c_int32), ("y", ctypes.c_int32), ("z", ctypes.c_int32),
                    ("found", ctypes.c_int32), ("score", ctypes.c_double), ("orientation", ctypes.c_int32),
                    ("diag", ctypes.c_uint32), ("n_candidates", ctypes.c_int32), ("err_ratio", ctypes.c_float)]

    def pack(k):
        t = ctypes.c_void_p()
        assert lib.psb_tray_create(*shape, ctypes.byref(t)) == 0, abi.err()
        assert lib.psb_tray_set(t, tray0.ctypes.data, None) == 0, abi.err()
        res = (Res * len(items))()
        out = np.zeros_like(tray0)
        lib.psb_debug_fail_alloc(k)
        st = lib.psb_pack(t, ptrs, dims.ctypes.data, len(items), maps.ctypes.data, 4, 1, 0, res, out.ctypes.data)
        lib.psb_debug_fail_alloc(0)
        msg = abi.err()
        assert lib.psb_tray_destroy(t) == 0
        return st, msg, res, out

    failures = 0
    for k in range(1, 160):
        st, msg, res, out = pack(k)
        assert abi.live() == base, k
        if st == 0:
            break
        assert st == PSB_ERR_CUDA and "injected" in msg, (k, st, msg)
        failures += 1
    assert failures >= 3
    st, _, res, out = pack(0)
    assert st == 0
    # the same placements as staging everything first (the oracle for this
    # 70-item run is minutes of CPU; the staged path is oracle-checked elsewhere)
    t = ctypes.c_void_p()
    assert lib.psb_tray_create(*shape, ctypes.byref(t)) == 0
    assert lib.psb_tray_set(t, tray0.ctypes.data, None) == 0
    lib.psb_pack_stage.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
    assert lib.psb_pack_stage(t, ptrs, dims.ctypes.data, len(items)) == 0, abi.err()
    res2 = (Res * len(items))()
    out2 = np.zeros_like(tray0)
    lib.psb_pack_staged.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int32,
                                    ctypes.c_void_p, ctypes.c_void_p]
    assert lib.psb_pack_staged(t, maps.ctypes.data, 4, 1, 0, res2, out2.ctypes.data) == 0, abi.err()
    assert lib.psb_tray_destroy(t) == 0
    np.testing.assert_array_equal(out, out2)
    assert [(r.found, r.x, r.y, r.z, r.orientation, r.score) for r in res] == \
           [(r.found, r.x, r.y, r.z, r.orientation, r.score) for r in res2]
