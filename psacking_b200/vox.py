"""Result export in the reference's .slab.vox layout (packing.cpp:274-305).

Header: three little-endian int32 sizes (x, y, z).  Body: one palette byte per
voxel, x from high to low, y from low to high, z from high to low; a voxel
value v (taken modulo 256, as the reference stores it in an unsigned char) is
written as 123 + v % 5 when non-zero (123 when v == 8, the voxelizer's INSIDE
flag) and 255 when empty.  Trailer: a 256-entry RGB palette with entries
123..127 set.
"""
from __future__ import annotations

import numpy as np

_PALETTE = np.zeros((256, 3), dtype=np.uint8)
_PALETTE[123] = (127, 0, 127)
_PALETTE[124] = (255, 0, 0)
_PALETTE[125] = (0, 255, 0)
_PALETTE[126] = (0, 0, 255)
_PALETTE[127] = (255, 255, 255)


def encode_vox(grid) -> bytes:
    g = np.asarray(grid)
    if g.ndim != 3:
        raise RuntimeError(f"Input array must be 3-dimensional, got {g.ndim}D")
    v = (g.astype(np.int64) & 0xFF).astype(np.uint8)
    pal = np.where(v != 0, 123 + (v % 5), 255).astype(np.uint8)
    pal[v == 8] = 123
    body = pal[::-1, :, ::-1]
    head = np.asarray(g.shape, dtype="<i4").tobytes()
    return head + np.ascontiguousarray(body).tobytes() + _PALETTE.tobytes()


def save_vox(grid, path: str) -> None:
    with open(path, "wb") as f:
        f.write(encode_vox(grid))
