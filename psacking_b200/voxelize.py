"""Mesh voxelization on the GPU: the reference's `voxelize_stl`
(spectral_packing/bindings.cpp:285-302; packing.cpp:540-588, VoxSurf).

`voxelize_stl(path, resolution)` reads a binary or ASCII STL file and
returns the tight int32 {0,1} grid of the mesh's surface voxels, the longest
side spanning `resolution` voxels (with the reference's 5 % margin).  The
rasterization runs in psb_voxelize_mesh (include/psb200.h).
"""
from __future__ import annotations

import ctypes
import struct
from pathlib import Path
from typing import Union

import numpy as np


def read_stl(path: Union[str, Path]) -> np.ndarray:
    """Triangles of an STL file as float32 [n, 3, 3] (vertex, xyz)."""
    data = Path(path).read_bytes()
    if len(data) >= 84:
        n = struct.unpack_from("<I", data, 80)[0]
        if len(data) == 84 + 50 * n:
            rec = np.frombuffer(data, dtype=np.dtype([("nrm", "<f4", 3), ("v", "<f4", (3, 3)), ("attr", "<u2")]),
                                count=n, offset=84)
            return np.ascontiguousarray(rec["v"], np.float32)
    text = data.decode("ascii", errors="replace").split()
    if not text or text[0] != "solid":
        raise RuntimeError(f"Failed to load mesh from: {path}")
    verts = [text[i + 1:i + 4] for i, tok in enumerate(text) if tok == "vertex"]
    if len(verts) % 3:
        raise RuntimeError(f"Failed to load mesh from: {path} (vertex count not a multiple of 3)")
    return np.asarray(verts, np.float32).reshape(-1, 3, 3)


def write_stl(path: Union[str, Path], tris: np.ndarray) -> None:
    """Binary STL (normals zero)."""
    tris = np.asarray(tris, np.float32).reshape(-1, 3, 3)
    rec = np.zeros(len(tris), dtype=np.dtype([("nrm", "<f4", 3), ("v", "<f4", (3, 3)), ("attr", "<u2")]))
    rec["v"] = tris
    Path(path).write_bytes(b"\0" * 80 + struct.pack("<I", len(tris)) + rec.tobytes())


def voxelize_mesh(tris: np.ndarray, resolution: int = 128) -> np.ndarray:
    from .proposal import check, lib
    tris = np.ascontiguousarray(np.asarray(tris, np.float32).reshape(-1, 3, 3))
    out = np.zeros(int(resolution) ** 3, np.int32)
    dims = np.zeros(3, np.int32)
    L = lib()
    L.psb_voxelize_mesh.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    check(L.psb_voxelize_mesh(tris.ctypes.data, len(tris), int(resolution), out.ctypes.data, dims.ctypes.data))
    n = int(np.prod(dims))
    if n == 0:  # make_voxel_grid_tight raises on a grid without occupied cells (voxelGrid.cpp:166-170)
        raise RuntimeError("(make_voxel_grid_tight) Voxel grid doesn't have any occupied cells")
    return out[:n].reshape(tuple(int(d) for d in dims)).copy()


def voxelize_stl(path: Union[str, Path], resolution: int = 128) -> np.ndarray:
    """bindings.cpp:285-302: load, voxelize, make tight."""
    try:
        return voxelize_mesh(read_stl(path), resolution)
    except Exception as e:  # the reference's message
        raise RuntimeError(f"Voxelization failed for {path}: {e}") from e
