"""CPU oracle for the placement search -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may import
this module, and only as the checker.  The product path (psacking_b200) never
calls it.

It restates the reference's per-item placement search (Vrroom/psacking) in
exact arithmetic: every correlation is an exact integer (direct sums for small
grids, FP64 FFTs rounded with a checked margin for large ones), so the answers
are what the reference computes when its FP32 cuFFT noise does not flip a
decision.  Each function cites the reference file:line it follows.

Pinning: tests/test_oracle_golden.py checks this module against every
known-answer vector in the reference's own tests (tests/golden/ref_kats.json,
generated by tests/golden/make_golden.py from the reference test sources).
"""
from __future__ import annotations

import math
from fractions import Fraction

import numpy as np

try:  # scipy's pocketfft runs FP64 FFTs multi-threaded; numpy's is the fallback
    import scipy.fft as _fft

    def _rfftn(a, s, workers):
        return _fft.rfftn(a, s=s, workers=workers)

    def _irfftn(a, s, workers):
        return _fft.irfftn(a, s=s, workers=workers)

    def _next_fast(n):
        return _fft.next_fast_len(int(n), real=True)
except ImportError:  # pragma: no cover
    def _rfftn(a, s, workers):
        return np.fft.rfftn(a, s=s)

    def _irfftn(a, s, workers):
        return np.fft.irfftn(a, s=s)

    def _next_fast(n):
        return int(n)

# spectral_packing/constants.h:7, :21 ; fft3.cu:161, :1361
P = 100000000.0
INF = 1000000000
INVALID = 1e30
FOUND_CUT = 1e29
WORKERS = -1  # scipy: all cores


def as_grid(a) -> np.ndarray:
    """numpy -> C-contiguous int32 3-D grid, as pybind11's
    array_t<int, c_style|forcecast> does (bindings.cpp:72-78, 129-135)."""
    g = np.ascontiguousarray(np.asarray(a).astype(np.int32, copy=False))
    if g.ndim != 3:
        raise RuntimeError(f"Input array must be 3-dimensional, got {g.ndim}D")
    return g


def bounds(g: np.ndarray):
    """get_voxel_grid_bounds (voxelGrid.cpp:279-299): lo/hi of voxels > 0,
    (INF,INF,INF)/(-INF,-INF,-INF) for an empty grid."""
    idx = np.argwhere(g > 0)
    if len(idx) == 0:
        return (INF, INF, INF), (-INF, -INF, -INF)
    lo = tuple(int(v) for v in idx.min(axis=0))
    hi = tuple(int(v) for v in idx.max(axis=0))
    return lo, hi


def make_tight(g):
    """make_voxel_grid_tight (voxelGrid.cpp:225-238)."""
    g = as_grid(g)
    lo, hi = bounds(g)
    if hi[0] == -INF:
        raise ValueError("(make_voxel_grid_tight) Voxel grid doesn't have any occupied cells")
    return np.ascontiguousarray(g[lo[0]:hi[0] + 1, lo[1]:hi[1] + 1, lo[2]:hi[2] + 1])


def pad_to(a: np.ndarray, shape) -> np.ndarray:
    """padto3d_flat (voxelGrid.cpp:262-276): zero-pad the array to shape."""
    out = np.zeros(shape, dtype=np.int64)
    out[:a.shape[0], :a.shape[1], :a.shape[2]] = a
    return out


# ----------------------------------------------------------------------------
# exact correlation
# ----------------------------------------------------------------------------

def corr_direct(tray: np.ndarray, item: np.ndarray) -> np.ndarray:
    """c[t] = sum_x item[x] * tray[t+x], tray zero outside its box, for every
    t in the tray's index box.  Exact integer arithmetic.

    This is what dft_corr3(tray, item) computes (packing.cpp:215-229: flip,
    convolve on the (2n+1)^3 grid, truncate, flip back) when its FP32 result
    rounds correctly."""
    T = tray.astype(np.int64)
    out = np.zeros(T.shape, dtype=np.int64)
    nx, ny, nz = T.shape
    for (x, y, z) in np.argwhere(item != 0):
        if x >= nx or y >= ny or z >= nz:
            continue
        v = int(item[x, y, z])
        out[:nx - x, :ny - y, :nz - z] += v * T[x:, y:, z:]
    return out


def corr_fft64(tray: np.ndarray, item: np.ndarray, linear: bool = True) -> np.ndarray:
    """Same quantity as corr_direct via FP64 FFTs, rounded to int64.

    linear=True pads to >= 2n-1 per axis (exact for every t).  linear=False
    uses a grid >= n per axis, which is exact only for translations where the
    whole item stays inside the tray -- the only ones the search scores.
    The rounding margin is checked: FP64 errors here are ~1e-7 absolute."""
    T = tray.astype(np.float64)
    shape = T.shape
    I = np.zeros(shape, dtype=np.float64)
    ex, ey, ez = (min(item.shape[a], shape[a]) for a in range(3))
    I[:ex, :ey, :ez] = item[:ex, :ey, :ez]
    if linear:
        s = tuple(_next_fast(2 * n - 1) for n in shape)
    else:
        s = tuple(_next_fast(n) for n in shape)
    FT = _rfftn(T, s, WORKERS)
    FI = _rfftn(I, s, WORKERS)
    c = _irfftn(np.conj(FI) * FT, s, WORKERS)[:shape[0], :shape[1], :shape[2]]
    r = np.rint(c)
    err = float(np.max(np.abs(c - r))) if c.size else 0.0
    if err > 0.05:
        raise AssertionError(f"FP64 correlation not exact (max rounding residue {err})")
    return r.astype(np.int64)


def corr_exact(tray, item, linear=True) -> np.ndarray:
    tray = np.asarray(tray)
    item = np.asarray(item)
    work = int(np.count_nonzero(item)) * tray.size
    if work <= 30_000_000:
        return corr_direct(tray, item)
    return corr_fft64(tray, item, linear=linear)


def dft_conv3(a, b) -> np.ndarray:
    """dft_conv3 (fft3.cu:643-715): linear convolution truncated to a's shape."""
    a, b = as_grid(a), as_grid(b)
    if a.shape != b.shape:
        raise RuntimeError("Input grids must be of the same size for convolution")
    # conv(a,b)[q] = sum_x a[x] b[q-x]  ==  corr(flip(b) placed ..) -- use direct
    n = a.shape
    out = np.zeros(n, dtype=np.int64)
    A = a.astype(np.int64)
    for (x, y, z) in np.argwhere(b != 0):
        v = int(b[x, y, z])
        out[x:, y:, z:] += v * A[:n[0] - x, :n[1] - y, :n[2] - z]
    return out.astype(np.int32)


def dft_corr3(a, b) -> np.ndarray:
    """dft_corr3 (packing.cpp:215-229): out[t] = sum_x b[x] a[t+x]."""
    a, b = as_grid(a), as_grid(b)
    if a.shape != b.shape:
        raise RuntimeError("Input grids must be of the same size for convolution")
    return corr_exact(a, b).astype(np.int32)


def collision_grid(tray, item) -> np.ndarray:
    """collision_grid (packing.cpp:241-252; binding pads the item to the tray
    shape, bindings.cpp:360-372): correlation, then out-of-tray positions
    raised to max(c, 1)."""
    tray, item = as_grid(tray), as_grid(item)
    padded = pad_to(item, tray.shape)
    _, hi = bounds(padded)
    c = corr_exact(tray, padded)
    nx, ny, nz = tray.shape
    i, j, k = np.indices(tray.shape)
    oob = ~((i + hi[0] <= nx - 1) & (j + hi[1] <= ny - 1) & (k + hi[2] <= nz - 1))
    c[oob] = np.maximum(c[oob], 1)
    return c.astype(np.int32)


# ----------------------------------------------------------------------------
# distance field
# ----------------------------------------------------------------------------

def calculate_distance(grid) -> np.ndarray:
    """calculate_distance, GPU build (fft3.cu:944-1004): sources are voxels
    EQUAL to 1 (fft3.cu:948); far value nx+ny+nz+10; one forward+backward
    min(d, d_nbr + 1) sweep per axis, x then y then z (= exact L1 distance)."""
    g = as_grid(grid)
    nx, ny, nz = g.shape
    far = nx + ny + nz + 10
    d = np.where(g == 1, 0, far).astype(np.int64)
    for axis in range(3):
        d = np.moveaxis(d, axis, 0).copy()
        n = d.shape[0]
        for s in range(n - 2, -1, -1):
            np.minimum(d[s], d[s + 1] + 1, out=d[s])
        for s in range(1, n):
            np.minimum(d[s], d[s - 1] + 1, out=d[s])
        d = np.moveaxis(d, 0, axis)
    return np.ascontiguousarray(d).astype(np.int32)


# ----------------------------------------------------------------------------
# flood fill (Algorithm 3)
# ----------------------------------------------------------------------------

def flood_reach(free: np.ndarray, exit_ijk) -> np.ndarray:
    """Cells of `free` 6-connected (through free cells) to a seed.  Seeds are
    the free cells on the faces i=0, j=0, k=0, i=exit_i, j=exit_j, k=exit_k
    (fft3.cu:263-293); propagation as fft3.cu:296-334 run to its fixed point.
    (The reference stops after nx+ny+nz sweeps, fft3.cu:437; reach_depth()
    reports when that cap would matter.)"""
    from scipy import ndimage

    nx, ny, nz = free.shape
    seed = np.zeros_like(free, dtype=bool)
    seed[0, :, :] = True
    seed[:, 0, :] = True
    seed[:, :, 0] = True
    ei, ej, ek = exit_ijk
    if 0 <= ei < nx:
        seed[ei, :, :] = True
    if 0 <= ej < ny:
        seed[:, ej, :] = True
    if 0 <= ek < nz:
        seed[:, :, ek] = True
    seed &= free
    st = ndimage.generate_binary_structure(3, 1)
    lab, n = ndimage.label(free, structure=st)
    hit = np.zeros(n + 1, dtype=bool)
    hit[np.unique(lab[seed])] = True
    hit[0] = False
    return hit[lab]


def reach_depth(free: np.ndarray, exit_ijk) -> int:
    """BFS depth (number of propagation steps) of the flood fill; the
    reference's in-place sweeps converge within this many iterations."""
    nx, ny, nz = free.shape
    reach = np.zeros_like(free, dtype=bool)
    reach[0], reach[:, 0], reach[:, :, 0] = free[0], free[:, 0], free[:, :, 0]
    ei, ej, ek = exit_ijk
    if 0 <= ei < nx:
        reach[ei] |= free[ei]
    if 0 <= ej < ny:
        reach[:, ej] |= free[:, ej]
    if 0 <= ek < nz:
        reach[:, :, ek] |= free[:, :, ek]
    depth = 0
    while True:
        grow = reach.copy()
        grow[1:] |= reach[:-1]
        grow[:-1] |= reach[1:]
        grow[:, 1:] |= reach[:, :-1]
        grow[:, :-1] |= reach[:, 1:]
        grow[:, :, 1:] |= reach[:, :, :-1]
        grow[:, :, :-1] |= reach[:, :, 1:]
        grow &= free
        if (grow == reach).all():
            return depth
        reach = grow
        depth += 1


def _valid_box(shape, hi):
    nx, ny, nz = shape
    return (min(nx, nx - hi[0]), min(ny, ny - hi[1]), min(nz, nz - hi[2]))


def interlocking_free_positions(tray, obj) -> np.ndarray:
    """interlocking_free_positions (bindings.cpp:561-648): obj_max from voxels
    != 0 (0 when empty), collision via collision_grid, labels/seeds/flood fill
    as fft3.cu:234-402."""
    tray, obj = as_grid(tray), as_grid(obj)
    nz_idx = np.argwhere(obj != 0)
    omax = tuple(int(v) for v in nz_idx.max(axis=0)) if len(nz_idx) else (0, 0, 0)
    coll = collision_grid(tray, obj)
    nx, ny, nz = tray.shape
    i, j, k = np.indices(tray.shape)
    oob = (i + omax[0] >= nx) | (j + omax[1] >= ny) | (k + omax[2] >= nz)
    free = (coll == 0) & ~oob
    ex = (max(0, nx - 1 - omax[0]), max(0, ny - 1 - omax[1]), max(0, nz - 1 - omax[2]))
    return flood_reach(free, ex).astype(np.int32)


# ----------------------------------------------------------------------------
# scores, tie rules, search
# ----------------------------------------------------------------------------

def fma_exact(a: float, b: float, c: float) -> float:
    """Correctly rounded a*b+c (IEEE fma) in pure Python."""
    return float(Fraction(a) * Fraction(b) + Fraction(c))


def score_scan(prox: int, k: int, nz: int) -> float:
    """packing.cpp:630-631: proximity + P * pow(k/L, 3.0) (host double)."""
    return float(prox) + P * math.pow(k / nz, 3.0)


def score_block(prox: int, k: int, nz: int) -> float:
    """fft3.cu:172-173: (double)prox + height_penalty*qz*qz*qz, whose last
    multiply and add nvcc contracts into one fma (default --fmad=true)."""
    qz = float(k) / float(nz)
    return fma_exact((P * qz) * qz, qz, float(prox))


def bitrev8(x: int) -> int:
    return int('{:08b}'.format(x & 255)[::-1], 2)


_BITREV8 = np.array([int('{:08b}'.format(v)[::-1], 2) for v in range(256)], dtype=np.int64)


def block_keys(idx: np.ndarray) -> np.ndarray:
    """block_key over an array of linear indices."""
    idx = np.asarray(idx, dtype=np.int64)
    return (idx & ~np.int64(255)) | _BITREV8[idx & 255]


def block_key(idx: int) -> int:
    """Tie order of argmin_reduction_kernel (fft3.cu:527-563) + the host finish
    (fft3.cu:1352-1357): lowest 256-block first (strict < over blocks), then
    inside a block the tree `if (s[t+s] < s[t])` keeps the lower slot on ties
    at every stride 128..1, i.e. the offset with the smallest bit-reversal."""
    return (idx & ~255) | bitrev8(idx & 255)


class TraySpectra:
    """FP64 half spectra of one tray state (binary occupancy and phi) on the
    circular grid s >= n per axis, computed once and shared by every
    orientation searched against that state.  The reference keeps the tray's
    spectra on the device between orientations the same way
    (GPUTrayContext::initialize, fft3.cu:1106-1175).  The occupancy has the
    same zero set of correlations as the reference's ID-valued tray for
    non-negative ids, and its counts are small enough to round exactly."""

    def __init__(self, tray, phi):
        tray, phi = as_grid(tray), as_grid(phi)
        self.shape = tray.shape
        self.s = tuple(_next_fast(n) for n in self.shape)
        self.occ = _rfftn((tray > 0).astype(np.float64), self.s, WORKERS)
        self.phi = _rfftn(phi.astype(np.float64), self.s, WORKERS)
        self.tray = tray
        self.phi_grid = phi

    def corr(self, spec_item, which):
        c = _irfftn(np.conj(spec_item) * (self.occ if which == "occ" else self.phi), self.s,
                    WORKERS)[:self.shape[0], :self.shape[1], :self.shape[2]]
        r = np.rint(c)
        err = float(np.max(np.abs(c - r))) if c.size else 0.0
        if err > 0.05:
            raise AssertionError(f"FP64 correlation not exact (max rounding residue {err})")
        return r.astype(np.int64)


def _search_fields(item, tray, phi, interlock, spectra=None):
    """Collision, proximity and the candidate mask of one orientation.

    With `spectra` (a TraySpectra of this tray and phi) the FFT correlations
    reuse the tray's spectra and the item's spectrum is computed once for both
    fields; the proximity is then computed only when some translation is a
    candidate (prox is None otherwise).  Results are identical on the cells
    the search reads: the valid box, where the circular correlation is exact."""
    nx, ny, nz = tray.shape
    padded = pad_to(item, tray.shape)
    _, hi = bounds(padded)
    Xv, Yv, Zv = _valid_box(tray.shape, hi)
    valid = np.zeros(tray.shape, dtype=bool)
    if Xv > 0 and Yv > 0 and Zv > 0:
        valid[:Xv, :Yv, :Zv] = True
    lin = False
    big = int(np.count_nonzero(padded)) * tray.size > 30_000_000
    if spectra is not None and big:
        FI = _rfftn(padded.astype(np.float64), spectra.s, WORKERS)
        coll = spectra.corr(FI, "occ")
        prox = None
    else:
        FI = None
        coll = corr_exact(tray, padded, linear=lin)
        prox = corr_exact(phi, padded, linear=lin)
    ok = valid & (coll == 0)
    if interlock and ok.any():
        ex = (nx - 1 - hi[0], ny - 1 - hi[1], nz - 1 - hi[2])
        ex = tuple(max(0, e) for e in ex)
        ok = flood_reach(ok, ex)
    if prox is None and ok.any():
        prox = spectra.corr(FI, "phi")
    return ok, prox


def search_one(item, tray, phi, mode="block", interlock=False, spectra=None):
    """One orientation: ((x,y,z), found, score).

    mode="scan"  -> fft_search_placement scoring (packing.cpp:590-642)
    mode="block" -> search_on_gpu / search_on_gpu_interlocking_free
                    (fft3.cu:1299-1459)."""
    item = as_grid(item)
    tray = as_grid(tray)
    phi = as_grid(phi)
    nx, ny, nz = tray.shape
    ok, prox = _search_fields(item, tray, phi, interlock, spectra)
    cand = np.flatnonzero(ok.ravel())
    if len(cand) == 0:
        return (-1, -1, -1), False, 0.0
    k = cand % nz
    pr = prox.ravel()[cand]
    if mode == "scan":
        pen = np.array([P * math.pow(kk / nz, 3.0) for kk in range(nz)])
        s = pr.astype(np.float64) + pen[k]
        best = int(np.argmin(s))          # first (lowest linear index) minimum
        if not s[best] < INF:
            return (-1, -1, -1), False, 0.0
        idx = int(cand[best])
        sc = float(s[best])
    else:
        qz = k.astype(np.float64) / float(nz)
        approx = pr.astype(np.float64) + ((P * qz) * qz) * qz
        m = approx.min()
        near = np.flatnonzero(approx <= m + abs(m) * 1e-14 + 1e-300)
        # exact scores of the near-minimal cells, once per distinct (prox, k)
        pk = np.stack([pr[near].astype(np.int64), k[near].astype(np.int64)], axis=1)
        uniq, inv = np.unique(pk, axis=0, return_inverse=True)
        sc_u = np.array([score_block(int(p), int(kk), nz) for p, kk in uniq])
        sc_n = sc_u[np.ravel(inv)]
        sc = float(sc_n.min())
        tied = cand[near[sc_n == sc]]
        idx = int(tied[int(np.argmin(block_keys(tied)))])
        if not sc < FOUND_CUT:
            return (-1, -1, -1), False, 0.0
    i, rem = divmod(idx, ny * nz)
    j, kk = divmod(rem, nz)
    return (int(i), int(j), int(kk)), True, sc


def fft_search_placement(item, tray):
    """fft_search_placement (bindings.cpp:182-203 -> packing.cpp:590-642)."""
    item, tray = as_grid(item), as_grid(tray)
    if any(item.shape[a] > tray.shape[a] for a in range(3)):
        return (-1, -1, -1), False, 0.0
    phi = calculate_distance(tray)
    return search_one(item, tray, phi, mode="scan")


def fft_search_placement_with_cache(item, tray, tray_distance, generation=0):
    """fft_search_placement_with_cache (bindings.cpp:220-247 -> fft3.cu:1506-1521)."""
    item = as_grid(item)
    tray = as_grid(tray)
    if any(item.shape[a] > tray.shape[a] for a in range(3)):
        return (-1, -1, -1), False, 0.0
    return search_one(item, tray, tray_distance, mode="block")


def fft_search_batch(orientations, tray, tray_distance, generation=0, interlock=False, spectra=None):
    """fft_search_batch / _interlocking_free (fft3.cu:1549-1632): orientations
    larger than the tray are skipped; strict < keeps the first best."""
    tray = as_grid(tray)
    best = ((-1, -1, -1), False, 1e30, -1)
    for o, it in enumerate(orientations):
        it = as_grid(it)
        if any(it.shape[a] > tray.shape[a] for a in range(3)):
            continue
        pos, found, sc = search_one(it, tray, tray_distance, mode="block", interlock=interlock, spectra=spectra)
        if found and sc < best[2]:
            best = (pos, True, sc, o)
    if not best[1]:
        return (-1, -1, -1), False, 1e30 if not interlock else 1e30, -1
    return best


def place_in_tray(item, tray, position, item_id=1):
    """place_in_tray (packing.cpp:773-788): copy; item voxels > 0 written as
    item_id where the tray is 0; RuntimeError at the first (row-major) tray
    cell where both are > 0.  Item parts outside the tray are ignored."""
    item, tray = as_grid(item), as_grid(tray)
    out = tray.copy()
    a, b, c = (int(v) for v in position)
    nx, ny, nz = tray.shape
    ex, ey, ez = item.shape
    i0, j0, k0 = max(a, 0), max(b, 0), max(c, 0)
    i1, j1, k1 = min(nx, a + ex), min(ny, b + ey), min(nz, c + ez)
    if i0 >= i1 or j0 >= j1 or k0 >= k1:
        return out
    sub_t = out[i0:i1, j0:j1, k0:k1]
    sub_i = item[i0 - a:i1 - a, j0 - b:j1 - b, k0 - c:k1 - c]
    clash = np.argwhere((sub_t > 0) & (sub_i > 0))
    if len(clash):
        i, j, k = clash[0] + np.array([i0, j0, k0])
        raise RuntimeError(
            "(place_in_tray): Item to be placed intersects with contents of tray at position "
            f"({i}, {j}, {k})")
    w = (sub_t == 0) & (sub_i > 0)
    sub_t[w] = item_id
    return out


# ----------------------------------------------------------------------------
# orientations (spectral_packer/rotations.py:141-219) and the packing loop
# ----------------------------------------------------------------------------

def _rx(g):
    return np.rot90(g, k=1, axes=(1, 2))


def _ry(g):
    return np.rot90(g, k=1, axes=(2, 0))


def _rz(g):
    return np.rot90(g, k=1, axes=(0, 1))


def orientations(grid, n=1):
    """get_orientations (rotations.py:222-272): 6 up-faces x 4 z-turns."""
    if n == 1:
        return [grid]
    if n == 4:
        out, g = [], grid.copy()
        for _ in range(4):
            out.append(g.copy())
            g = _rz(g)
        return out
    if n == 6:
        return [grid, _rx(grid), _rx(_rx(grid)), _rx(_rx(_rx(grid))), _ry(grid), _ry(_ry(_ry(grid)))]
    if n == 24:
        faces = [grid, _rx(grid), _rx(_rx(grid)), _rx(_rx(_rx(grid))), _ry(grid), _ry(_ry(_ry(grid)))]
        out = []
        for f in faces:
            g = f.copy()
            for _ in range(4):
                out.append(g.copy())
                g = _rz(g)
        return out
    raise ValueError(f"num_orientations must be 1, 4, 6, or 24, got {n}")


def pack_voxels(items, tray_size, num_orientations=1, interlocking_free=False,
                sort_by_volume=True, initial_tray=None, fast=False, progress=None):
    """BinPacker.pack_voxels (packer.py:366-544) over the oracle searches.
    Returns (tray, placements) with placements as dicts in original order.

    fast=True shares each tray state's spectra between the orientations of an
    item (TraySpectra); the answers are the same.  progress(n_done, placement)
    is called after every item when given."""
    proc = [np.asarray(it).astype(np.int32) for it in items]
    vols = [int(np.sum(it > 0)) for it in proc]
    if sort_by_volume:
        order = list(np.argsort(vols)[::-1])
    else:
        order = list(range(len(items)))
    if initial_tray is not None:
        tray = np.asarray(initial_tray).astype(np.int32).copy()
        id_offset = int(np.max(tray))
    else:
        tray = np.zeros(tray_size, dtype=np.int32)
        id_offset = 0
    placements = []
    num_placed = 0
    for orig in order:
        item = proc[orig]
        best = (None, float("inf"), 0, item)
        found_any = False
        ors = orientations(item, num_orientations)
        spectra = None
        if num_orientations > 1 or interlocking_free:
            phi = calculate_distance(tray)
            if fast:
                spectra = TraySpectra(tray, phi)
        if interlocking_free:
            valid, vidx = [], []
            for o, r in enumerate(ors):
                r = np.ascontiguousarray(r.astype(np.int32))
                if not any(r.shape[a] > tray_size[a] for a in range(3)):
                    valid.append(r)
                    vidx.append(o)
            if valid:
                pos, found, sc, bo = fft_search_batch(valid, tray, phi, interlock=True, spectra=spectra)
                if found and bo >= 0:
                    best = (pos, sc, vidx[bo], valid[bo])
                    found_any = True
        else:
            for o, r in enumerate(ors):
                r = np.ascontiguousarray(r.astype(np.int32))
                if any(r.shape[a] > tray_size[a] for a in range(3)):
                    continue
                if num_orientations > 1:
                    pos, found, sc = search_one(r, tray, phi, mode="block", spectra=spectra)
                else:
                    pos, found, sc = fft_search_placement(r, tray)
                if found and sc < best[1]:
                    best = (pos, sc, o, r)
                    found_any = True
        if found_any:
            tray = place_in_tray(best[3], tray, best[0], id_offset + num_placed + 1)
            num_placed += 1
            placements.append(dict(item_index=int(orig), position=tuple(best[0]), score=best[1],
                                   success=True, volume=vols[orig], orientation_index=best[2]))
        else:
            placements.append(dict(item_index=int(orig), position=None, score=None,
                                   success=False, volume=vols[orig], orientation_index=0))
        if progress is not None:
            progress(len(placements), placements[-1])
    placements.sort(key=lambda p: p["item_index"])
    return tray, placements


def density(tray) -> float:
    """BinPacker._calculate_stats (packer.py:582-601): occupied / bbox volume."""
    occ = tray > 0
    n = int(occ.sum())
    if n == 0:
        return 0.0
    idx = np.argwhere(occ)
    dims = idx.max(axis=0) - idx.min(axis=0) + 1
    return float(n / np.prod(dims))
