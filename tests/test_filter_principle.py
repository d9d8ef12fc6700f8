"""The candidate pre-filter's exactness argument and word arithmetic, on the
CPU (no GPU call).

The packing loop's pre-filter (psacking_b200/csrc/psb_filter.cuh) keeps, per
(x, y) column of translations, the z bits where a sample S of the item's
voxels lands on empty tray cells.  Three facts make it safe, checked here
against the oracle's exact collision count (oracle/psb_oracle.py corr_direct,
the reference's collision_grid semantics):
  * every collision-free translation is a candidate, for ANY sample subset
    (the filter may stop sampling early), and with all voxels sampled the
    candidates are exactly the free translations;
  * the direct check of k_cand_verify (item columns as two mask words against
    shifted tray words) is exactly "collision count == 0";
  * the kernel's word arithmetic (tray columns as 32-bit words, a sample at
    height s.z shifting by s.z // 32 whole words and a funnel shift of
    s.z % 32) gives the same bits as the plain boolean definition.
"""
import numpy as np
import pytest

from oracle import psb_oracle as O


def free_translations(tray, item):
    """Boolean [Xv, Yv, Zv]: collision-free translations (count == 0)."""
    hi = np.argwhere(item > 0).max(axis=0)
    c = O.corr_direct((tray != 0).astype(np.int64), (item > 0).astype(np.int64))
    Xv, Yv, Zv = (np.array(tray.shape) - hi)
    return c[:Xv, :Yv, :Zv] == 0


def candidates(tray, item, samples):
    """Boolean [Xv, Yv, Zv]: translations where every sample lands on an
    empty cell (the filter's definition)."""
    hi = np.argwhere(item > 0).max(axis=0)
    Xv, Yv, Zv = (np.array(tray.shape) - hi)
    empty = tray == 0
    cand = np.ones((Xv, Yv, Zv), bool)
    for sx, sy, sz in samples:
        cand &= empty[sx:sx + Xv, sy:sy + Yv, sz:sz + Zv]
    return cand


def words_of(col_bits, nw):
    """Bit list along z -> nw little-endian 32-bit words."""
    w = [0] * nw
    for z, b in enumerate(col_bits):
        if b:
            w[z >> 5] |= 1 << (z & 31)
    return w


def funnel_r(lo, hi, off):
    return (((hi << 32) | lo) >> off) & 0xFFFFFFFF


def candidates_words(tray, item, samples):
    """The same candidates through the kernel's word arithmetic (k_cand_filter:
    c[w] &= funnel(T[w + k], T[w + k + 1]) >> off, k = s.z // 32)."""
    hi = np.argwhere(item > 0).max(axis=0)
    nx, ny, nz = tray.shape
    Xv, Yv, Zv = (nx - hi[0], ny - hi[1], nz - hi[2])
    nw = 4 * ((((nz + 31) // 32) + 3) // 4)   # words per tray column (uint4 granules)
    T = {(i, j): words_of(tray[i, j] == 0, nw) for i in range(nx) for j in range(ny)}
    out = np.zeros((Xv, Yv, Zv), bool)
    for x in range(Xv):
        for y in range(Yv):
            c = [(0xFFFFFFFF if Zv - 32 * w >= 32 else ((1 << max(0, Zv - 32 * w)) - 1)) for w in range(nw)]
            for sx, sy, sz in samples:
                sx, sy, sz = int(sx), int(sy), int(sz)   # Python ints: no 64-bit wrap in the shifts
                col = T[(x + sx, y + sy)]
                k, off = sz >> 5, sz & 31
                for w in range(nw):
                    lo = col[w + k] if w + k < nw else 0
                    hi_w = col[w + k + 1] if w + k + 1 < nw else 0
                    c[w] &= funnel_r(lo, hi_w, off)
            for z in range(Zv):
                out[x, y, z] = (c[z >> 5] >> (z & 31)) & 1
    return out


def random_case(rng, shape, fill):
    tray = (rng.random(shape) < fill).astype(np.int32) * rng.integers(1, 5, shape).astype(np.int32)
    e = rng.integers(2, 6, 3)
    item = (rng.random(tuple(e)) < 0.6).astype(np.int32)
    item[0, 0, 0] = 1
    item[e[0] - 1, e[1] - 1, e[2] - 1] = 1
    return tray, item


@pytest.mark.parametrize("seed", range(6))
def test_any_sample_subset_keeps_every_free_translation(seed):
    rng = np.random.default_rng(seed)
    tray, item = random_case(rng, (12, 11, 40), 0.15)
    free = free_translations(tray, item)
    vox = [tuple(int(c) for c in v) for v in np.argwhere(item > 0)]
    for m in (1, 3, 8, len(vox)):
        pick = rng.choice(len(vox), size=m, replace=False)
        cand = candidates(tray, item, [vox[i] for i in pick])
        assert not (free & ~cand).any()           # free is a subset of the candidates
    assert np.array_equal(candidates(tray, item, vox), free)   # all voxels: exactly the free set


@pytest.mark.parametrize("seed,nz", [(0, 20), (1, 40), (2, 70), (3, 100), (4, 150)])
def test_word_arithmetic_matches_the_boolean_definition(seed, nz):
    """Columns of 20..150 cells, so samples shift by 0..4 whole words,
    candidates straddle word boundaries, and columns of more than 128 cells
    take two 16-byte granules (the kernel's NQ = 2 form, eight words)."""
    rng = np.random.default_rng(100 + seed)
    tray, item = random_case(rng, (7, 6, nz), 0.1)
    h = nz - 3                                   # samples up to z = nz - 4: shifts of up to 4 words
    item = np.zeros((3, 2, h), np.int32)
    item[0, 0, 0] = item[2, 1, -1] = item[1, 0, h // 2] = 1
    for z in (31, 32, 63, 64, 127, 128):         # samples on word boundaries
        if z < h:
            item[z % 3, z % 2, z] = 1
    vox = [tuple(int(c) for c in v) for v in np.argwhere(item > 0)]
    got = candidates_words(tray, item, vox)
    assert np.array_equal(got, candidates(tray, item, vox))
    assert np.array_equal(got, free_translations(tray, item))


def verify_columns(tray, item, x, y, z):
    """k_cand_verify's test of one translation: item column (a, b) as two
    mask words (bits c < 32, 32 <= c < 64); tray column (x + a, y + b) as
    empty-cell words; free when no mask bit meets a non-empty cell of
    funnel(T[z // 32 + j], T[z // 32 + j + 1]) >> z % 32."""
    nx, ny, nz = tray.shape
    nzw = (nz + 31) // 32
    for a in range(item.shape[0]):
        for b in range(item.shape[1]):
            col = item[a, b] > 0
            if not col.any():
                continue
            m = words_of(col, 2)
            T = words_of(tray[x + a, y + b] == 0, nzw)
            sh, off = z >> 5, z & 31
            t0 = T[sh]
            t1 = T[sh + 1] if sh + 1 < nzw else 0
            t2 = T[sh + 2] if sh + 2 < nzw else 0
            f0 = funnel_r(t0, t1, off)
            f1 = funnel_r(t1, t2, off) if m[1] else 0
            if (m[0] & ~f0 & 0xFFFFFFFF) | (m[1] & ~f1 & 0xFFFFFFFF):
                return False
    return True


@pytest.mark.parametrize("seed,nz", [(0, 40), (1, 70), (2, 100)])
def test_direct_column_check_matches_the_collision_count(seed, nz):
    """Items up to 64 cells high (two mask words), translations across word
    boundaries: the direct check is exactly "collision count == 0"."""
    rng = np.random.default_rng(200 + seed)
    tray = (rng.random((9, 8, nz)) < 0.08).astype(np.int32)
    h = min(nz - 4, 60)
    item = (rng.random((3, 3, h)) < 0.15).astype(np.int32)
    item[0, 0, 0] = item[2, 2, h - 1] = 1
    free = free_translations(tray, item)
    Xv, Yv, Zv = free.shape
    got = np.array([[[verify_columns(tray, item, x, y, z) for z in range(Zv)] for y in range(Yv)]
                    for x in range(Xv)])
    assert np.array_equal(got, free)
