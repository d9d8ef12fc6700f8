"""GPU parity: the CUDA path against the CPU oracle and the golden fixture.

Every comparison is exact: positions, found flags and scores (doubles) must be
bit-identical to the oracle, which is the reference's algorithm in exact
arithmetic.  Run on a B200 with `pytest -m gpu`."""
import ctypes
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from oracle import psb_oracle as O
from tests.golden_io import load_records, same_output

pytestmark = pytest.mark.gpu

HERE = Path(__file__).resolve().parent
SCAN, BLOCK, INTERLOCK = 0, 1, 0x10
DIAG_FALSE_FREE, DIAG_BOUND = 0x4, 0x8


# --------------------------------------------------------------------------
# golden replay through the drop-in module
# --------------------------------------------------------------------------
RECORDS = load_records()


def _replay(core, r):
    a = r["args"]
    fn = r["fn"]
    if fn == "fft_search_batch":
        core.gpu_tray_cleanup()
        return core.fft_search_batch(list(a[0]), a[1], a[2], 1)
    if fn == "fft_search_placement_with_cache":
        core.gpu_tray_cleanup()
        return core.fft_search_placement_with_cache(a[0], a[1], a[2], 1)
    if fn == "place_in_tray":
        return core.place_in_tray(a[0], a[1], a[2], a[3])
    if fn == "pack_voxels":
        from psacking_b200 import BinPacker
        items, tray_size, n_orient, interlock, sort = a[:5]
        initial = a[5] if len(a) > 5 else None
        outs = []
        for engine in ("native", "calls"):
            res = BinPacker(tuple(tray_size), num_orientations=n_orient, interlocking_free=interlock,
                            engine=engine).pack_voxels(list(items), sort_by_volume=sort, initial_tray=initial)
            outs.append((res.tray, [(p.position, p.success, p.orientation_index, p.score) for p in res.placements]))
        assert same_output(outs[0], outs[1])
        return outs[0]
    return getattr(core, fn)(*a)


@pytest.mark.parametrize("i", range(len(RECORDS)))
def test_golden_replay(gpu_core, i):
    r = RECORDS[i]
    got = _replay(gpu_core, r)
    assert same_output(got, r["out"]), (r["test"], r["fn"])


# --------------------------------------------------------------------------
# per-orientation search parity on random trays
# --------------------------------------------------------------------------
def random_tray(rng, shape, fill, with_first_item=True):
    tray = np.zeros(shape, np.int32)
    n = int(fill * np.prod(shape) / 30) + 1
    for b in range(n):
        e = [int(rng.integers(1, max(2, s // 4) + 1)) for s in shape]
        o = [int(rng.integers(0, s - ee + 1)) for s, ee in zip(shape, e)]
        tray[o[0]:o[0] + e[0], o[1]:o[1] + e[1], o[2]:o[2] + e[2]] = 1 + (b if not with_first_item else b + 1) % 7
    return tray


def random_item(rng, maxe):
    e = [int(rng.integers(1, m + 1)) for m in maxe]
    it = (rng.random(e) < 0.7).astype(np.int32)
    if it.sum() == 0:
        it[tuple(np.array(e) - 1)] = 1
    return it


def check_search(core, tray, items, flags, phi=None):
    if phi is None:
        phi = O.calculate_distance(tray)
    core.gpu_tray_init(tray, phi)
    d = core.search_detail(items, flags)
    mode = "scan" if (flags & 0xF) == SCAN else "block"
    inter = bool(flags & INTERLOCK)
    best = None
    for o, it in enumerate(items):
        pos, found, score, diag, ncand, err_ratio = d["per_orientation"][o]
        assert err_ratio <= 1.0
        assert not diag & (DIAG_FALSE_FREE | DIAG_BOUND), (o, hex(diag))
        if any(it.shape[a] > tray.shape[a] for a in range(3)):
            assert not found
            continue
        want = O.search_one(it, tray, phi, mode=mode, interlock=inter)
        assert (tuple(pos), found) == (tuple(want[0]), want[1]), (o, pos, want)
        if found:
            assert score == want[2], (o, score, want[2])
            if best is None or score < best[1]:
                best = (o, score, tuple(pos))
    bpos, bfound, bscore, bo = d["best"]
    if best is None:
        assert not bfound
    else:
        assert bfound and bo == best[0] and bscore == best[1] and tuple(bpos) == best[2]


SHAPES = [(9, 7, 8), (17, 23, 19), (32, 32, 32), (40, 33, 27), (64, 64, 64)]


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("flags", [SCAN, BLOCK, BLOCK | INTERLOCK])
def test_search_random(gpu_core, shape, flags):
    rng = np.random.default_rng(hash((shape, flags)) % 2**32)
    for trial in range(3):
        tray = random_tray(rng, shape, [0.0, 0.15, 0.4][trial])
        items = [random_item(rng, [max(1, s // 3) for s in shape]) for _ in range(4)]
        check_search(gpu_core, tray, items, flags)


def test_search_padded_grid(gpu_core):
    """A 90x70x110 tray is padded to the specialised lengths 100x100x128
    (within twice the smooth lengths' volume): the circular correlation on
    the longer grid must still give the oracle's exact answers."""
    import ctypes
    from psacking_b200.proposal import lib
    shape = (90, 70, 110)
    t = ctypes.c_void_p()
    L = lib()
    assert L.psb_tray_create(*shape, ctypes.byref(t)) == 0
    F = (ctypes.c_int * 3)()
    assert L.psb_tray_fft_dims(t, F) == 0
    L.psb_tray_destroy(t)
    assert tuple(F) == (100, 100, 128)
    rng = np.random.default_rng(41)
    for flags in (BLOCK | INTERLOCK, BLOCK, SCAN):
        tray = random_tray(rng, shape, 0.3)
        items = [random_item(rng, [12, 10, 14]) for _ in range(3)]
        check_search(gpu_core, tray, items, flags)


def test_padded_grid_packing(gpu_core):
    from psacking_b200 import workloads
    run_both(workloads.config2_items(21)[:8], (90, 70, 110), 6, True)


def test_search_empty_and_full(gpu_core):
    tray = np.zeros((20, 20, 20), np.int32)
    it = np.ones((3, 3, 3), np.int32)
    check_search(gpu_core, tray, [it], BLOCK)
    check_search(gpu_core, tray, [it], SCAN)
    full = np.ones((6, 6, 6), np.int32)
    check_search(gpu_core, full, [it], BLOCK | INTERLOCK)
    big = np.ones((25, 3, 3), np.int32)
    check_search(gpu_core, tray, [big, it], BLOCK)


DIAG_FLOOD_FILL = 0x400


def caged_tray(hole):
    """A sealed box (walls of id 2, thickness 2) whose cavity holds the only
    distance source (a voxel equal to 1): the best free cell for a 5^3 item is
    inside the cavity.  hole: None (sealed), "offset" (a roof opening away
    from the source: reachable only by a bent path) or "above" (an opening
    straight above the best cell)."""
    tray = np.zeros((40, 40, 100), np.int32)
    tray[4:24, 4:24, 0:16] = 2
    tray[6:22, 6:22, 1:14] = 0
    tray[14, 14, 1] = 1
    if hole == "offset":
        tray[16:22, 16:22, 14:16] = 0
    elif hole == "above":
        tray[6:22, 6:22, 14:16] = 0
    return tray


@pytest.mark.parametrize("variant", [3, 2])
@pytest.mark.parametrize("hole", [None, "offset", "above"])
def test_caged_interlock_search(gpu_core, hole, variant):
    """A cavity whose best free cell is sealed, reachable by a bent path, or
    by a straight one: the answer is the oracle's (sealed: the winner moves
    outside; otherwise it stays inside).  Variant 3 (default) always runs the
    flood fill before the proximity pass; variant 2 runs it lazily, only when
    the best free cell has no straight free run to a seed face."""
    gpu_core.set_plane_variant(variant)
    tray = caged_tray(hole)
    phi = O.calculate_distance(tray)
    item = np.ones((5, 5, 5), np.int32)
    ors = [item, np.ones((3, 5, 7), np.int32)]
    want = O.fft_search_batch(ors, tray, phi, interlock=True)
    gpu_core.gpu_tray_init(tray, phi)
    try:
        d = gpu_core.search_detail(ors, BLOCK | INTERLOCK, per_orientation=False)
    finally:
        gpu_core.set_plane_variant(3)
    pos, found, score, bo = d["best"]
    assert (tuple(pos), found, score, bo) == (tuple(want[0]), want[1], want[2], want[3])
    if variant == 2:
        ran = bool(d["best_diag"] & DIAG_FLOOD_FILL)
        assert ran == (hole != "above"), hex(d["best_diag"])
    inside = 6 <= pos[0] < 22 and 6 <= pos[1] < 22 and 1 <= pos[2] < 14
    assert inside == (hole is not None)
    got = gpu_core.fft_search_batch_interlocking_free(ors, tray, phi, 1)
    assert (tuple(got[0]), got[1], got[2], got[3]) == (tuple(want[0]), want[1], want[2], want[3])


@pytest.fixture(params=["fast", "share", "plane2", "generic"])
def fft_variant(request, gpu_core):
    gpu_core.set_fast_fft(request.param != "generic")
    gpu_core.set_plane_variant(2 if request.param == "plane2" else 3)
    gpu_core.set_share_flips(request.param == "share")
    yield request.param
    gpu_core.set_fast_fft(True)
    gpu_core.set_plane_variant(3)
    gpu_core.set_share_flips(False)


def test_search_config3_scale(gpu_core, fft_variant):
    """240x123x100 tray (the benchmark's tray), two large items, 24 orientations
    of one of them, interlocking mask on: exact parity at full size."""
    from psacking_b200 import workloads
    from psacking_b200.rotations import get_orientations
    rng = np.random.default_rng(11)
    shape = workloads.TRAY3
    tray = np.zeros(shape, np.int32)
    tray[0:60, 0:50, 0:40] = 1
    tray[100:150, 60:123, 0:30] = 2
    tray[30:200, 20:40, 40:60] = 3
    items = workloads.config3_items(5, n=2)
    ors = [np.ascontiguousarray(o) for o in get_orientations(items[0], 24)][::4] + [items[1]]
    check_search(gpu_core, tray, ors, BLOCK | INTERLOCK)
    check_search(gpu_core, tray, ors[:2], BLOCK)


# --------------------------------------------------------------------------
# distance, correlation, flood fill at sizes the oracle handles quickly
# --------------------------------------------------------------------------
@pytest.mark.parametrize("shape", [(1, 1, 1), (1000, 1, 1), (1, 1, 700), (33, 1, 65), (64, 64, 64), (240, 123, 100)])
def test_distance(gpu_core, shape):
    rng = np.random.default_rng(sum(shape))
    g = (rng.random(shape) < 0.001).astype(np.int32)
    g[rng.random(shape) < 0.01] = 3
    assert np.array_equal(gpu_core.calculate_distance(g), O.calculate_distance(g))
    assert np.array_equal(gpu_core.calculate_distance(np.zeros(shape, np.int32)),
                          O.calculate_distance(np.zeros(shape, np.int32)))


@pytest.mark.parametrize("shape", [(5, 6, 7), (16, 16, 16), (31, 20, 9)])
def test_corr_conv(gpu_core, shape):
    rng = np.random.default_rng(shape[0])
    a = rng.integers(0, 6, shape).astype(np.int32)
    b = rng.integers(0, 3, shape).astype(np.int32)
    assert np.array_equal(gpu_core.dft_corr3(a, b), O.dft_corr3(a, b))
    assert np.array_equal(gpu_core.dft_conv3(a, b), O.dft_conv3(a, b))
    item = (rng.random((3, 4, 2)) < 0.6).astype(np.int32)
    assert np.array_equal(gpu_core.collision_grid(a, item), O.collision_grid(a, item))
    tray = (rng.random(shape) < 0.3).astype(np.int32)
    assert np.array_equal(gpu_core.interlocking_free_positions(tray, item),
                          O.interlocking_free_positions(tray, item))


def test_place_in_tray(gpu_core):
    tray = np.zeros((6, 5, 4), np.int32)
    tray[2, 2, 2] = 9
    it = np.ones((2, 2, 2), np.int32)
    out = gpu_core.place_in_tray(it, tray, (0, 0, 0), 5)
    assert np.array_equal(out, O.place_in_tray(it, tray, (0, 0, 0), 5))
    with pytest.raises(RuntimeError, match=r"position \(2, 2, 2\)"):
        gpu_core.place_in_tray(it, tray, (1, 1, 1), 5)
    # clipped at the tray edge like the reference loop
    out = gpu_core.place_in_tray(it, tray, (5, 4, 3), 7)
    assert np.array_equal(out, O.place_in_tray(it, tray, (5, 4, 3), 7))


# --------------------------------------------------------------------------
# whole packing runs: identical placements, trays and densities
# --------------------------------------------------------------------------
def run_both(items, tray_size, n_orient, interlock):
    from psacking_b200 import BinPacker
    out = {}
    for engine in ("native", "calls"):
        r = BinPacker(tray_size, num_orientations=n_orient, interlocking_free=interlock,
                      engine=engine).pack_voxels(items)
        out[engine] = r
    want_tray, want_pl = O.pack_voxels(items, tray_size, n_orient, interlock)
    for engine, r in out.items():
        assert np.array_equal(r.tray, want_tray), engine
        for p, w in zip(r.placements, want_pl):
            assert (p.success, p.position, p.orientation_index) == (w["success"], w["position"],
                                                                   w["orientation_index"]), engine
            if p.success:
                assert p.score == w["score"]
        assert r.density == O.density(want_tray)
    return out


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_config1_packing(gpu_core, seed, fft_variant):
    from psacking_b200 import workloads
    run_both(workloads.config1_items(seed), workloads.TRAY1, 1, False)


def test_config2_prefix_packing(gpu_core, fft_variant):
    from psacking_b200 import workloads
    items = workloads.config2_items(100)[:6]
    run_both(items, workloads.TRAY2, 24, False)


def test_config3_prefix_packing(gpu_core, fft_variant):
    from psacking_b200 import workloads
    items = workloads.config3_items(100)[:3]
    run_both(items, workloads.TRAY3, 24, True)


def test_small_interlock_packing(gpu_core):
    from psacking_b200 import workloads
    items = workloads.config1_items(7)[:12]
    run_both(items, (40, 40, 12), 4, True)
    run_both(items, (40, 40, 12), 6, False)


# --------------------------------------------------------------------------
# the score expression of the reference as nvcc evaluates it
# --------------------------------------------------------------------------
def test_reference_score_expression_is_fused(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    so = tmp_path / "probe.so"
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-Xcompiler", "-fPIC",
                    "-o", str(so), str(HERE / "probes" / "score_probe.cu")], check=True)
    lib = ctypes.CDLL(str(so))
    rng = np.random.default_rng(0)
    n = 4096
    prox = rng.integers(0, 3_000_000, n).astype(np.int32)
    nz = 100
    k = rng.integers(0, nz, n).astype(np.int32)
    out = np.zeros(n, np.float64)
    P = ctypes.POINTER
    rc = lib.run_score_probe(prox.ctypes.data_as(P(ctypes.c_int)), k.ctypes.data_as(P(ctypes.c_int)),
                             ctypes.c_int(nz), ctypes.c_double(1e8), out.ctypes.data_as(P(ctypes.c_double)),
                             ctypes.c_int(n))
    assert rc == 0
    fused = np.array([O.score_block(int(p), int(kk), nz) for p, kk in zip(prox, k)])
    assert np.array_equal(out, fused)


# --------------------------------------------------------------------------
# many independent trays (concurrent streams) == one run per tray
# --------------------------------------------------------------------------
def test_pack_many_matches_single_runs(gpu_core):
    from psacking_b200 import BinPacker, workloads
    rng = np.random.default_rng(3)
    trays = []
    for t in range(5):
        dims = tuple(int(v) for v in rng.integers(40, 90, 3))
        trays.append((dims, workloads.config2_items(500 + t, n=int(rng.integers(4, 9)))))
    for n_orient, inter in [(4, True), (1, False), (24, False)]:
        p = BinPacker((8, 8, 8), num_orientations=n_orient, interlocking_free=inter)
        many = p.pack_many(trays, concurrency=3)
        for (dims, items), r in zip(trays, many):
            one = BinPacker(dims, num_orientations=n_orient, interlocking_free=inter).pack_voxels(items)
            assert np.array_equal(r.tray, one.tray)
            assert [(q.position, q.orientation_index, q.score) for q in r.placements] == \
                   [(q.position, q.orientation_index, q.score) for q in one.placements]


# --------------------------------------------------------------------------
# orientation sharding of one tray (one rank here: the same code path that
# several ranks run, with the decision exchange reduced to the identity)
# --------------------------------------------------------------------------
@pytest.mark.parametrize("cfg", ["config2", "config3"])
def test_orientation_sharded_packing_matches(gpu_core, cfg):
    from psacking_b200 import BinPacker, workloads
    from psacking_b200.shard import pack_orientation_sharded
    if cfg == "config2":
        items, tray, n, inter = workloads.config2_items(11)[:8], (96, 96, 96), 24, False
    else:
        items, tray, n, inter = workloads.config3_items(12)[:4], workloads.TRAY3, 24, True
    ref = BinPacker(tray, num_orientations=n, interlocking_free=inter).pack_voxels(items)
    got_tray, got = pack_orientation_sharded(items, tray, n, inter)
    assert np.array_equal(got_tray, ref.tray)
    for p, g in zip(ref.placements, got):
        assert (p.success, p.position, p.orientation_index) == (g[0], g[1], g[2] if g[0] else 0)
        if p.success:
            assert p.score == g[3]


# --------------------------------------------------------------------------
# candidate pre-filter of the packing loop: same results with and without it
# --------------------------------------------------------------------------
def _detail_run(items, tray_size, interlock):
    from psacking_b200 import proposal as PR
    from psacking_b200.rotations import orientation_maps
    seq = PR.sorted_by_volume(items)
    tray = PR.Tray(tray_size)
    try:
        res, per, _, final = tray.pack_detail(seq, orientation_maps(24), interlock)
    finally:
        tray.close()
    key = lambda r: (r.found, r.x, r.y, r.z, r.score)  # noqa: E731
    direct = sum(1 for r in per if r.diag & 0x800)
    return [key(r) + (r.orientation,) for r in res], [key(r) for r in per], final, direct


@pytest.mark.parametrize("case", ["config2-free", "config3-interlock", "config3-generic", "config3-plane2"])
def test_cand_filter_same_results(gpu_core, case):
    """Trays that fill up, so the filter skips orientations and planes and
    decides orientations with few candidates directly: the placements, every
    orientation's own result and the final tray are the same with the filter
    off, on with every sample and no direct decisions, and on with the
    defaults (sampling cut-off, direct decisions)."""
    from psacking_b200 import workloads
    # (100, 64, 64): every axis has a specialised FFT length, so the default
    # search takes the split flow that decides orientations directly
    if case == "config2-free":
        items, dims, il = workloads.config2_items(3)[:60], (100, 64, 64), False
    else:
        items, dims, il = workloads.config3_items(9)[:40], (100, 64, 64), True
    gpu_core.set_fast_fft(case != "config3-generic")
    gpu_core.set_plane_variant(2 if case == "config3-plane2" else 3)
    try:
        gpu_core.set_cand_filter(False)
        want = _detail_run(items, dims, il)
        gpu_core.set_cand_filter(True)
        gpu_core.set_direct_max(0)
        gpu_core.set_filter_cut(0)       # every sample tested
        mid = _detail_run(items, dims, il)
        gpu_core.set_direct_max(4096)
        gpu_core.set_filter_cut(50)      # the defaults
        got = _detail_run(items, dims, il)
    finally:
        gpu_core.set_cand_filter(True)
        gpu_core.set_direct_max(4096)
        gpu_core.set_filter_cut(50)
        gpu_core.set_fast_fft(True)
        gpu_core.set_plane_variant(3)
    for run in (mid, got):
        assert run[0] == want[0]
        assert run[1] == want[1]
        assert np.array_equal(run[2], want[2])
    placed = sum(r[0] for r in want[0])
    assert 0 < placed < len(items)   # the tray filled up: the filter had work to skip
    assert want[3] == 0 and mid[3] == 0
    if case in ("config2-free", "config3-interlock"):
        assert got[3] > 0            # some orientations were decided directly
    else:
        assert got[3] == 0           # only the split flow decides directly


def test_cand_filter_full_tray_against_oracle(gpu_core):
    """A small tray packed until items stop fitting, against the oracle, in
    both modes (the filter is on by default)."""
    from psacking_b200 import workloads
    items = workloads.config1_items(4)
    run_both(items, (30, 30, 14), 6, True)
    run_both(items, (30, 30, 14), 6, False)
