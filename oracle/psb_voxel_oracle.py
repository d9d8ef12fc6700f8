"""CPU oracle of the mesh voxelizer (test infrastructure).

A restatement of the reference's voxelize_stl path for triangle meshes:
  spectral_packing/bindings.cpp:285-302   load, voxelize, make tight
  spectral_packing/packing.cpp:309-335    isInTriangle: 64-bit edge functions
                                          at the pixel centre, barycentric depth
  spectral_packing/packing.cpp:337-410    rasterize along the three axes
                                          (swizzles xyz, yzx, zxy), XOR of the
                                          axis bit per hit, aligned-edge rule
  spectral_packing/packing.cpp:540-588    voxelize: exact vertex merge, the
                                          box transform in float32, rounding,
                                          resolution, rasterization; no inside
                                          fill (constants.h:9 VOXEL_FILL_INSIDE 0)
  LibSL Mesh.cpp:350-392                  mergeVerticesExact: new index = rank
                                          of the position in lexicographic order
  LibSL Matrix4x4.h:245-294               float32 matrix product and mulPoint,
                                          accumulated from zero in index order
Pinned against the reference's own voxelize_stl (its module compiled from
its sources by oracle/Makefile): tests/golden/make_voxel_golden.py records
its outputs on seeded meshes in tests/golden/ref_voxels.npz, which this
restatement reproduces bit for bit (tests/test_voxel_oracle.py).  Only tests
import it.
"""
from __future__ import annotations

import numpy as np

FP_POW = 16
FP_SCALE = 1 << FP_POW
ALONG_X, ALONG_Y, ALONG_Z = 1, 2, 4
f32 = np.float32


def merge_vertices_exact(tris: np.ndarray):
    """tris [n, 3, 3] float32 -> (positions [m, 3] in lexicographic order,
    triangle indices [n, 3])."""
    v = np.asarray(tris, np.float32).reshape(-1, 3)
    order = np.lexsort((np.arange(len(v)), v[:, 2], v[:, 1], v[:, 0]))
    sv = v[order]
    new = np.empty(len(v), np.int64)
    idx = -1
    prev = None
    for k, o in enumerate(order):
        p = tuple(sv[k])
        if p != prev:
            idx += 1
        new[o] = idx
        prev = p
    pos = np.zeros((idx + 1, 3), np.float32)
    pos[new] = v
    return pos, new.reshape(-1, 3)


def _mat_mul(a, b):
    r = np.zeros((4, 4), np.float32)
    for i in range(4):
        for j in range(4):
            acc = f32(0)
            for k in range(4):
                acc = f32(acc + f32(a[i, k] * b[k, j]))
            r[i, j] = acc
    return r


def _scale(s):
    m = np.eye(4, dtype=np.float32)
    for i in range(3):
        m[i, i] = f32(s[i])
    return m


def _translate(t):
    m = np.eye(4, dtype=np.float32)
    for i in range(3):
        m[i, 3] = f32(t[i])
    return m


def box_transform(pos: np.ndarray, resolution: int):
    """(integer fixed-point vertices [m, 3], voxel grid dims)."""
    lo = pos.min(axis=0).astype(np.float32)
    hi = pos.max(axis=0).astype(np.float32)
    ext = (hi - lo).astype(np.float32)
    emax = f32(ext.max())
    factor = f32(0.95)
    s1 = _scale([f32(resolution * FP_SCALE)] * 3)
    s2 = _scale([f32(f32(1.0) / emax)] * 3)
    t1 = _translate([f32(f32(f32(f32(1.0) - factor) * f32(0.5)) * ext[i]) for i in range(3)])
    s3 = _scale([factor] * 3)
    t2 = _translate([f32(-lo[i]) for i in range(3)])
    m = _mat_mul(_mat_mul(_mat_mul(_mat_mul(s1, s2), t1), s3), t2)
    top = f32(resolution * FP_SCALE) - f32(1.0)
    pts = np.zeros((len(pos), 3), np.int64)
    for p, v in enumerate(pos):
        for i in range(3):
            acc = f32(0)
            for k in range(3):
                acc = f32(acc + f32(m[i, k] * v[k]))
            acc = f32(acc + m[i, 3])
            r = np.round(acc) if acc != np.floor(acc) + f32(0.5) else (np.floor(acc) + 1 if acc >= 0 else np.ceil(acc) - 1)
            r = f32(min(max(f32(r), f32(0.0)), top))
            pts[p, i] = int(r)
    dims = [int(f32(f32(ext[i] / emax) * f32(resolution))) for i in range(3)]
    return pts, dims


def _in_triangle(i, j, p0, p1, p2):
    """packing.cpp:309-335 for one sample (i, j) in fixed point: (inside,
    depth, aligned)."""
    d0 = (i - p0[0], j - p0[1])
    d1 = (i - p1[0], j - p1[1])
    d2 = (i - p2[0], j - p2[1])
    e10 = (p1[0] - p0[0], p1[1] - p0[1])
    e21 = (p2[0] - p1[0], p2[1] - p1[1])
    e02 = (p0[0] - p2[0], p0[1] - p2[1])
    c0 = d0[0] * e10[1] - d0[1] * e10[0]
    c1 = d1[0] * e21[1] - d1[1] * e21[0]
    c2 = d2[0] * e02[1] - d2[1] * e02[0]
    inside = (c0 <= 0 and c1 <= 0 and c2 <= 0) or (c0 >= 0 and c1 >= 0 and c2 >= 0)
    aligned = 0 if c0 == 0 else (1 if c1 == 0 else (2 if c2 == 0 else -1))
    depth = 0
    if inside:
        area = c0 + c1 + c2

        def tdiv(a, b):  # C++ integer division truncates toward zero
            q = abs(a) // abs(b)
            return q if (a >= 0) == (b > 0) else -q
        b0 = tdiv(c1 << 10, area)
        b1 = tdiv(c2 << 10, area)
        b2 = (1 << 10) - b0 - b1
        depth = (b0 * p0[2] + b1 * p1[2] + b2 * p2[2]) >> 10
    return inside, depth, aligned


SWIZZLES = [  # (forward, backward, along)
    (lambda v: (v[0], v[1], v[2]), lambda v: (v[0], v[1], v[2]), ALONG_Z),
    (lambda v: (v[1], v[2], v[0]), lambda v: (v[2], v[0], v[1]), ALONG_X),
    (lambda v: (v[2], v[0], v[1]), lambda v: (v[1], v[2], v[0]), ALONG_Y),
]


def rasterize(tri, pts, vox):
    dims = vox.shape
    for fwd, bwd, along in SWIZZLES:
        tp = [fwd(tuple(int(c) for c in pts[tri[k]])) for k in range(3)]
        e10 = (tp[1][0] - tp[0][0], tp[1][1] - tp[0][1])
        e21 = (tp[2][0] - tp[1][0], tp[2][1] - tp[1][1])
        e02 = (tp[0][0] - tp[2][0], tp[0][1] - tp[2][1])
        if e10 == (0, 0) or e21 == (0, 0) or e02 == (0, 0):
            continue
        # the reference forms this determinant from int products (v2i), which
        # wrap modulo 2^32 at these fixed-point magnitudes: a triangle whose
        # determinant is a nonzero multiple of 2^32 is skipped as degenerate
        if (e02[0] * e10[1] - e02[1] * e10[0]) % (1 << 32) == 0:
            continue
        xs = [p[0] // FP_SCALE for p in tp]
        ys = [p[1] // FP_SCALE for p in tp]
        for j in range(min(ys), max(ys) + 1):
            for i in range(min(xs), max(xs) + 1):
                inside, depth, aligned = _in_triangle((i << FP_POW) + (1 << (FP_POW - 1)),
                                                      (j << FP_POW) + (1 << (FP_POW - 1)), tp[0], tp[1], tp[2])
                if not inside:
                    continue
                if aligned != -1 and not (tri[aligned] < tri[(aligned + 1) % 3]):
                    continue
                v = bwd((i, j, depth >> FP_POW))
                if all(0 <= v[a] < dims[a] for a in range(3)):
                    vox[v] ^= along


def make_tight(g: np.ndarray) -> np.ndarray:
    """voxelGrid.cpp:166-178: the bounding box of the occupied cells; an
    empty grid raises, as the reference does."""
    idx = np.argwhere(g > 0)
    if len(idx) == 0:
        raise RuntimeError("(make_voxel_grid_tight) Voxel grid doesn't have any occupied cells")
    lo, hi = idx.min(axis=0), idx.max(axis=0) + 1
    return g[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]]


def voxelize(tris: np.ndarray, resolution: int = 128) -> np.ndarray:
    """Surface voxels (any axis parity bit set), tight, int32 {0, 1}."""
    pos, idx = merge_vertices_exact(tris)
    pts, dims = box_transform(pos, resolution)
    vox = np.zeros(dims, np.int64)
    for t in idx:
        rasterize(t, pts, vox)
    return make_tight((vox > 0).astype(np.int32))
