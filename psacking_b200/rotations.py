"""Axis-aligned item orientations in the reference's order.

The order is part of the interface: `orientation_index` in a placement means
"the k-th array returned by get_orientations" (spectral_packer/rotations.py:
159-272).  The 24 orientations are 6 choices of the up face (identity, +x
quarter turns 1..3, +y quarter turn, +y three quarter turns) times 4 quarter
turns about z, each turn being numpy's rot90 on the same axis pair as the
reference (x: axes (1,2); y: axes (2,0); z: axes (0,1)).

`orientation_maps` turns that order into signed axis permutations, which the
device uses to gather every orientation from the single uploaded item.
"""
from __future__ import annotations

from typing import List

import numpy as np

_TURN_AXES = {"x": (1, 2), "y": (2, 0), "z": (0, 1)}
# up-face preludes, applied before the z turns (rotations.py:187-217)
_FACES = ("", "x", "xx", "xxx", "y", "yyy")
# the 6-orientation subset uses the same preludes without z turns (rotations.py:257-265)


def _turn(g: np.ndarray, axis: str) -> np.ndarray:
    return np.rot90(g, k=1, axes=_TURN_AXES[axis])


def rotate_90_x(grid: np.ndarray) -> np.ndarray:
    """Quarter turn about x (y -> z)."""
    return _turn(grid, "x")


def rotate_90_y(grid: np.ndarray) -> np.ndarray:
    """Quarter turn about y (z -> x)."""
    return _turn(grid, "y")


def rotate_90_z(grid: np.ndarray) -> np.ndarray:
    """Quarter turn about z (x -> y)."""
    return _turn(grid, "z")


def _prelude(grid: np.ndarray, face: str) -> np.ndarray:
    g = grid
    for a in face:
        g = _turn(g, a)
    return g


def get_24_orientations(grid: np.ndarray) -> List[np.ndarray]:
    out = []
    for face in _FACES:
        g = _prelude(grid, face)
        for _ in range(4):
            out.append(g.copy())
            g = rotate_90_z(g)
    return out


def get_orientations(grid: np.ndarray, num_orientations: int = 1) -> List[np.ndarray]:
    if num_orientations == 1:
        return [grid]
    if num_orientations == 4:
        return get_24_orientations(grid)[:4]
    if num_orientations == 6:
        return [_prelude(grid, f) for f in _FACES]
    if num_orientations == 24:
        return get_24_orientations(grid)
    raise ValueError(f"num_orientations must be 1, 4, 6, or 24, got {num_orientations}")


def make_contiguous(grid: np.ndarray) -> np.ndarray:
    return grid if grid.flags["C_CONTIGUOUS"] else np.ascontiguousarray(grid)


def orientation_maps(num_orientations: int) -> np.ndarray:
    """(n, 6) int32 rows [src_axis0, src_axis1, src_axis2, flip0, flip1, flip2]
    such that oriented[i0,i1,i2] = item[s] with
    s[src_axis[a]] = (e[a]-1-i[a]) if flip[a] else i[a].

    Derived by running get_orientations on a probe grid whose axes have
    distinct lengths and whose values are the linear source index."""
    b = (2, 3, 5)
    probe = np.arange(np.prod(b), dtype=np.int64).reshape(b)
    rows = []
    for g in get_orientations(probe, num_orientations):
        src = np.unravel_index(int(g[0, 0, 0]), b)
        axes, flips = [], []
        for a in range(3):
            s = b.index(g.shape[a])
            axes.append(s)
            flips.append(1 if src[s] == b[s] - 1 else 0)
        rows.append(axes + flips)
    return np.asarray(rows, dtype=np.int32)


def apply_map(item: np.ndarray, row) -> np.ndarray:
    """Host restatement of the device gather (for tests)."""
    axes, flips = list(row[:3]), list(row[3:])
    inv = [axes.index(s) for s in range(3)]
    g = np.transpose(item, axes)
    sl = tuple(slice(None, None, -1) if flips[a] else slice(None) for a in range(3))
    return np.ascontiguousarray(g[sl])


def _rotation_matrices() -> List[np.ndarray]:
    """The 24 orientations as rotation matrices on voxel-centre coordinates
    measured from the grid centre: a voxel at x in the item lands at R @ x
    in the oriented grid.  Row a of R holds one entry, at the source axis of
    output axis a (orientation_maps), -1 where that axis is reversed.  These
    equal the reference's ROTATION_MATRICES_3x3 (rotations.py:41-89), which
    blender export uses to turn a placement's orientation_index into a mesh
    transform."""
    out = []
    for row in orientation_maps(24):
        r = np.zeros((3, 3), dtype=np.float64)
        for a in range(3):
            r[a, int(row[a])] = -1.0 if row[3 + a] else 1.0
        out.append(r)
    return out


ROTATION_MATRICES_3x3: List[np.ndarray] = _rotation_matrices()


def get_rotation_matrix_3x3(orientation_index: int) -> np.ndarray:
    """3x3 rotation of orientation `orientation_index` (0..23, the order of
    get_24_orientations); IndexError outside that range (rotations.py:92-112)."""
    if not 0 <= orientation_index < 24:
        raise IndexError(f"orientation_index must be 0-23, got {orientation_index}")
    return ROTATION_MATRICES_3x3[orientation_index].copy()


def get_rotation_matrix_4x4(orientation_index: int) -> np.ndarray:
    """The same rotation as a 4x4 homogeneous matrix, no translation
    (rotations.py:115-138)."""
    m = np.eye(4, dtype=np.float64)
    m[:3, :3] = get_rotation_matrix_3x3(orientation_index)
    return m
