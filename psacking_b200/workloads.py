"""Seeded synthetic workloads standing in for the reference's datasets.

The reference measures density on Thingi10K meshes (README.md:12), which are
not available here.  These generators produce voxel items with the shapes,
sizes and value distributions of the benchmark configurations:

  config1: 64^3 tray, 20 items, unions of 1-3 boxes (extents 4-16) on a 16^3
           canvas, identity orientation only.
  config2: 128^3 tray, 100 items, half superellipsoids (semi-axes 4-20,
           exponents 0.3-3), half box unions (bounding box 8-40), 24 orientations.
  config3: 240x123x100 tray, 350 items of largest extent 20-50: superellipsoids
           (semi-axes 10-25), tori (major radius 8-20, minor 3-8) and U/L hooks
           (wall thickness 3-6), 24 orientations, interlocking-free.
  config5: 64 trays with sides drawn from 64..160, 50-300 config2-style items each.
"""
from __future__ import annotations

from typing import List, Tuple

import numpy as np

TRAY1 = (64, 64, 64)
TRAY2 = (128, 128, 128)
TRAY3 = (240, 123, 100)


def _tight(g: np.ndarray) -> np.ndarray:
    idx = np.argwhere(g > 0)
    if len(idx) == 0:
        return g.astype(np.int32)
    lo, hi = idx.min(axis=0), idx.max(axis=0) + 1
    return np.ascontiguousarray(g[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]]).astype(np.int32)


def box_union(rng, canvas: Tuple[int, int, int], n_boxes: int, emin: int, emax: int) -> np.ndarray:
    g = np.zeros(canvas, dtype=np.int32)
    for _ in range(n_boxes):
        e = [int(rng.integers(emin, min(emax, canvas[a]) + 1)) for a in range(3)]
        o = [int(rng.integers(0, canvas[a] - e[a] + 1)) for a in range(3)]
        g[o[0]:o[0] + e[0], o[1]:o[1] + e[1], o[2]:o[2] + e[2]] = 1
    return _tight(g)


def superellipsoid(a: float, b: float, c: float, e1: float, e2: float) -> np.ndarray:
    """Voxels whose centres satisfy (|x/a|^(2/e2) + |y/b|^(2/e2))^(e2/e1) + |z/c|^(2/e1) <= 1."""
    n = [2 * int(np.ceil(s)) for s in (a, b, c)]
    x = (np.arange(n[0]) + 0.5 - n[0] / 2) / a
    y = (np.arange(n[1]) + 0.5 - n[1] / 2) / b
    z = (np.arange(n[2]) + 0.5 - n[2] / 2) / c
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    f = (np.abs(X) ** (2 / e2) + np.abs(Y) ** (2 / e2)) ** (e2 / e1) + np.abs(Z) ** (2 / e1)
    return _tight((f <= 1.0).astype(np.int32))


def torus(R: float, r: float, axis: int) -> np.ndarray:
    s = int(np.ceil(R + r))
    h = int(np.ceil(r))
    x = np.arange(2 * s) + 0.5 - s
    z = np.arange(2 * h) + 0.5 - h
    X, Y, Z = np.meshgrid(x, x, z, indexing="ij")
    g = ((np.sqrt(X ** 2 + Y ** 2) - R) ** 2 + Z ** 2 <= r * r).astype(np.int32)
    if axis != 2:
        g = np.moveaxis(g, 2, axis)
    return _tight(g)


def hook(rng, kind: str) -> np.ndarray:
    """U or L profile (wall thickness 3-6) extruded along one axis."""
    t = int(rng.integers(3, 7))
    w = int(rng.integers(14, 41))
    h = int(rng.integers(14, 41))
    d = int(rng.integers(max(t, 6), 25))
    prof = np.zeros((w, h), dtype=np.int32)
    prof[:t, :] = 1
    prof[:, :t] = 1
    if kind == "U":
        prof[w - t:, :] = 1
    g = np.repeat(prof[:, :, None], d, axis=2)
    perm = rng.permutation(3)
    return _tight(np.transpose(g, perm))


def config1_items(seed: int, n: int = 20) -> List[np.ndarray]:
    rng = np.random.default_rng(seed)
    return [box_union(rng, (16, 16, 16), int(rng.integers(1, 4)), 4, 16) for _ in range(n)]


def config2_items(seed: int, n: int = 100) -> List[np.ndarray]:
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < n:
        if len(out) % 2 == 0:
            a, b, c = rng.uniform(4, 20, 3)
            e1, e2 = rng.uniform(0.3, 3, 2)
            it = superellipsoid(a, b, c, e1, e2)
        else:
            canvas = tuple(int(v) for v in rng.integers(8, 41, 3))
            it = box_union(rng, canvas, int(rng.integers(1, 4)), 4, 40)
        if it.size and it.sum() > 0:
            out.append(it)
    return out


def config3_items(seed: int, n: int = 350) -> List[np.ndarray]:
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < n:
        kind = int(rng.integers(0, 4))
        if kind == 0:
            a, b, c = rng.uniform(10, 25, 3)
            e1, e2 = rng.uniform(0.3, 3, 2)
            it = superellipsoid(a, b, c, e1, e2)
        elif kind == 1:
            it = torus(rng.uniform(8, 20), rng.uniform(3, 8), int(rng.integers(0, 3)))
        else:
            it = hook(rng, "U" if kind == 2 else "L")
        m = max(it.shape)
        if 20 <= m <= 50 and it.sum() > 0:
            out.append(it)
    return out


def config5_trays(seed: int, n_trays: int = 64):
    rng = np.random.default_rng(seed)
    trays = []
    for t in range(n_trays):
        dims = tuple(int(v) for v in rng.integers(64, 161, 3))
        n_items = int(rng.integers(50, 301))
        trays.append((dims, config2_items(seed * 1000 + t, n_items)))
    return trays


def volume(items) -> int:
    return int(sum(int((np.asarray(i) > 0).sum()) for i in items))
