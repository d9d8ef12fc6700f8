"""Generates tests/golden/ref_voxels.npz: the reference's own voxelize_stl on
seeded triangle meshes, the fixture that pins the voxelizer oracle
(oracle/psb_voxel_oracle.py) and the GPU voxelizer, and the SHA-256 of the
files its save_vox writes for seeded grids (packing.cpp:274-305), which pin
psacking_b200/vox.py.

    python tests/golden/make_voxel_golden.py <dir holding the reference's built spectral_packer>

The directory is the one `make -C oracle REF=<reference checkout>` fills
(oracle/_ref): the reference's pybind11 module compiled from its sources
(bindings.cpp:285-302 py_voxelize_stl, packing.cpp:309-588 voxelize), next to
its unmodified Python package.  Voxelization is CPU code in that module, so
this runs without a GPU.  Every case writes the mesh as a binary STL, calls
spectral_packer._core.voxelize_stl(path, resolution) and records the tight
int32 grid, or that the call raised (the reference raises when the grid has
no occupied cell, voxelGrid.cpp:166-170).
"""
from __future__ import annotations

import hashlib
import os
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from psacking_b200.voxelize import write_stl  # noqa: E402  (pure Python, no native code)
from tests import meshes  # noqa: E402


def _rotation(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    a, b, c, d = q
    return np.array([[a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
                     [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
                     [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d]])


def cases():
    """(name, float32 triangles [n, 3, 3], resolution)."""
    out = []
    # axis-aligned boxes: the unit cube at every resolution 8..64 in steps of 4
    # (at resolutions where 0.95 * res is an integer the reference's 32-bit
    # degeneracy test wraps to zero for every face: no voxel, an error)
    for res in range(8, 65, 4):
        out.append((f"cube-{res}", meshes.box(), res))
    for k, (hi, res) in enumerate([((2.0, 1.0, 0.3), 32), ((1.0, 3.0, 0.7), 40), ((0.5, 0.5, 2.0), 28),
                                   ((1.3, 1.7, 1.1), 48)]):
        out.append((f"box{k}-{res}", meshes.box(hi=hi), res))
    out.append(("tetra-32", meshes.tetra(), 32))
    out.append(("sphere2-32", meshes.icosphere(2), 32))
    out.append(("sphere1-20", meshes.icosphere(1) + np.float32(3.7), 20))
    out.append(("torus-48", meshes.torus(), 48))
    out.append(("torus-thin-40", meshes.torus(R=1.0, r=0.12, n=32, m=10), 40))
    # seeded rigid motions and anisotropic scales of the same shapes
    rng = np.random.default_rng(20240607)
    shapes = [("box", meshes.box()), ("tetra", meshes.tetra()), ("sphere", meshes.icosphere(2)),
              ("torus", meshes.torus(n=20, m=10))]
    for k in range(16):
        name, tris = shapes[k % len(shapes)]
        m = _rotation(rng) @ np.diag(rng.uniform(0.4, 2.0, 3))
        t = rng.uniform(-5, 5, 3)
        res = int(rng.choice([16, 24, 32, 40, 48, 64]))
        tt = (tris.reshape(-1, 3).astype(np.float64) @ m.T + t).astype(np.float32).reshape(-1, 3, 3)
        out.append((f"{name}-moved{k}-{res}", tt, res))
    return out


def main(ref_dir: str) -> None:
    sys.path.insert(0, str(Path(ref_dir).resolve()))
    import spectral_packer._core as R  # the reference's module, built from its sources

    rec = {}
    names = []
    with tempfile.TemporaryDirectory() as d:
        for name, tris, res in cases():
            p = os.path.join(d, "mesh.stl")
            write_stl(p, tris)
            names.append(name)
            rec[f"{name}/tris"] = np.asarray(tris, np.float32)
            rec[f"{name}/res"] = np.int32(res)
            try:
                g = np.asarray(R.voxelize_stl(p, res), np.int32)
            except RuntimeError:
                rec[f"{name}/error"] = np.int8(1)
                print(f"{name}: raised")
                continue
            assert set(np.unique(g)) <= {0, 1}
            rec[f"{name}/shape"] = np.asarray(g.shape, np.int32)
            rec[f"{name}/bits"] = np.packbits(g.astype(np.uint8).ravel())
            print(f"{name}: {g.shape} {int(g.sum())} voxels")
        # save_vox: seeded grids with empty cells, the INSIDE flag value 8,
        # values above 255 and negative values (stored modulo 256)
        rng = np.random.default_rng(7)
        for k in range(12):
            shape = tuple(int(v) for v in rng.integers(1, 14, 3))
            g = rng.integers(-3, 600, shape).astype(np.int32)
            g[rng.random(shape) < 0.4] = 0
            g[rng.random(shape) < 0.1] = 8
            p = os.path.join(d, "grid.slab.vox")
            R.save_vox(g, p)
            data = Path(p).read_bytes()
            rec[f"savevox/{k}/grid"] = g
            rec[f"savevox/{k}/sha256"] = np.asarray(hashlib.sha256(data).hexdigest())
            rec[f"savevox/{k}/nbytes"] = np.int64(len(data))
        rec["savevox_count"] = np.int32(12)
    rec["names"] = np.asarray(names)
    np.savez_compressed(ROOT / "tests" / "golden" / "ref_voxels.npz", **rec)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    main(sys.argv[1])
