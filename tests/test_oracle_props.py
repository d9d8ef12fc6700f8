"""Self-consistency of the CPU oracle (independent formulations agree)."""
import math
from collections import deque
from fractions import Fraction

import numpy as np
import pytest
from scipy import ndimage

from oracle import psb_oracle as O


def bfs_l1(grid):
    # multi-source BFS from voxels == 1; far value for unreachable as the GPU build
    far = sum(grid.shape) + 10
    d = np.full(grid.shape, far, np.int64)
    q = deque()
    for idx in zip(*np.nonzero(grid == 1)):
        d[idx] = 0
        q.append(idx)
    while q:
        x = q.popleft()
        for ax in range(3):
            for s in (-1, 1):
                y = list(x)
                y[ax] += s
                if 0 <= y[ax] < grid.shape[ax] and d[tuple(y)] > d[x] + 1:
                    d[tuple(y)] = d[x] + 1
                    q.append(tuple(y))
    return d


@pytest.mark.parametrize("seed", range(6))
def test_corr_direct_equals_fft64(seed):
    rng = np.random.default_rng(seed)
    shape = tuple(int(v) for v in rng.integers(3, 14, 3))
    T = rng.integers(0, 5, shape)
    I = np.zeros(shape, np.int64)
    e = [int(rng.integers(1, s + 1)) for s in shape]
    I[:e[0], :e[1], :e[2]] = rng.integers(0, 3, e)
    assert np.array_equal(O.corr_direct(T, I), O.corr_fft64(T, I, linear=True))
    # circular grid: exact wherever the item stays inside
    c = O.corr_fft64(T, I, linear=False)
    hi = [max(np.nonzero(I.any(axis=tuple(b for b in range(3) if b != a)))[0], default=0) for a in range(3)]
    d = O.corr_direct(T, I)
    v = tuple(slice(0, shape[a] - hi[a]) for a in range(3))
    assert np.array_equal(c[v], d[v])


@pytest.mark.parametrize("seed", range(5))
def test_distance_is_l1_bfs(seed):
    rng = np.random.default_rng(seed)
    shape = tuple(int(v) for v in rng.integers(1, 12, 3))
    g = (rng.random(shape) < [0.0, 0.02, 0.2, 0.5, 0.9][seed]).astype(np.int32)
    g[rng.random(shape) < 0.1] = 2  # ids >= 2 are not sources
    assert np.array_equal(O.calculate_distance(g), bfs_l1(g))


@pytest.mark.parametrize("seed", range(5))
def test_flood_matches_bfs(seed):
    rng = np.random.default_rng(seed)
    shape = (9, 7, 8)
    free = rng.random(shape) < 0.6
    ex = (6, 5, 4)
    r = O.flood_reach(free, ex)
    # plain BFS from the seed faces
    seen = np.zeros(shape, bool)
    q = deque()
    for idx in zip(*np.nonzero(free)):
        if idx[0] in (0, ex[0]) or idx[1] in (0, ex[1]) or idx[2] in (0, ex[2]):
            seen[idx] = True
            q.append(idx)
    while q:
        x = q.popleft()
        for ax in range(3):
            for s in (-1, 1):
                y = list(x)
                y[ax] += s
                y = tuple(y)
                if 0 <= y[ax] < shape[ax] and free[y] and not seen[y]:
                    seen[y] = True
                    q.append(y)
    assert np.array_equal(r, seen)
    assert O.reach_depth(free, ex) >= 0


def test_fma_exact_and_block_key():
    for a, b, c in [(0.1, 0.2, 0.3), (1e8 * 0.37 * 0.37, 0.37, 12345.0), (3.0, 1 / 3, -1.0)]:
        want = float(Fraction(a) * Fraction(b) + Fraction(c))
        assert O.fma_exact(a, b, c) == want
    assert O.bitrev8(1) == 128 and O.bitrev8(128) == 1 and O.bitrev8(255) == 255
    # offsets 0..255: the tree keeps even slots first, so offset 0 < 128 < 64 ...
    keys = sorted(range(256), key=O.block_key)
    assert keys[:4] == [0, 128, 64, 192]
    assert O.block_key(256) == 256


def test_tree_argmin_tie_rule_simulated():
    # simulate argmin_reduction_kernel (fft3.cu:527-563) on tied scores
    rng = np.random.default_rng(1)
    for _ in range(200):
        s = rng.integers(0, 3, 256).astype(float)
        idx = list(range(256))
        vals = list(s)
        st = 128
        while st > 0:
            for t in range(st):
                if vals[t + st] < vals[t]:
                    vals[t], idx[t] = vals[t + st], idx[t + st]
            st //= 2
        m = s.min()
        want = min((i for i in range(256) if s[i] == m), key=O.block_key)
        assert idx[0] == want


def test_scores():
    assert O.score_scan(5, 0, 10) == 5.0
    assert O.score_scan(0, 5, 10) == 1e8 * math.pow(0.5, 3.0)
    qz = 3 / 7
    assert O.score_block(11, 3, 7) == O.fma_exact((1e8 * qz) * qz, qz, 11.0)


def test_search_brute_force_small():
    rng = np.random.default_rng(7)
    for _ in range(20):
        shape = tuple(int(v) for v in rng.integers(4, 9, 3))
        tray = (rng.random(shape) < 0.25).astype(np.int32) * rng.integers(1, 4, shape).astype(np.int32)
        item = (rng.random(tuple(int(v) for v in rng.integers(1, 4, 3))) < 0.7).astype(np.int32)
        if item.sum() == 0:
            item[0, 0, 0] = 1
        phi = O.calculate_distance(tray)
        for mode in ("scan", "block"):
            pos, found, sc = O.search_one(item, tray, phi, mode=mode)
            # brute force
            best = None
            nx, ny, nz = shape
            hi = O.bounds(O.pad_to(item, shape))[1]
            for i in range(nx):
                for j in range(ny):
                    for k in range(nz):
                        if i + hi[0] > nx - 1 or j + hi[1] > ny - 1 or k + hi[2] > nz - 1:
                            continue
                        coll = prox = 0
                        for (a, b, c) in np.argwhere(item != 0):
                            coll += item[a, b, c] * tray[i + a, j + b, k + c]
                            prox += item[a, b, c] * phi[i + a, j + b, k + c]
                        if coll:
                            continue
                        s = O.score_scan(prox, k, nz) if mode == "scan" else O.score_block(prox, k, nz)
                        lin = (i * ny + j) * nz + k
                        key = (s, lin if mode == "scan" else O.block_key(lin))
                        if best is None or key < best[0]:
                            best = (key, (i, j, k))
            if best is None:
                assert not found
            else:
                assert found and pos == best[1] and sc == best[0][0]
