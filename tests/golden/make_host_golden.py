"""Generates tests/golden/ref_host.npz: outputs of the reference's own host
functions on seeded edge cases, the fixture that pins the oracle's
restatements of them (oracle/psb_oracle.py).

    python tests/golden/make_host_golden.py <dir holding the reference's built spectral_packer>

The directory is the one `make -C oracle REF=<reference checkout>` fills
(oracle/_ref).  The functions recorded run on the host in the reference's
module, so this needs no GPU:
  place_in_tray (bindings.cpp:259-276, packing.cpp:773-788): items partly or
      wholly outside the tray, negative positions, negative and zero values
      in item and tray, overlaps (the call raises; the message names the
      first overlapping cell in row-major order);
  make_tight / get_bounds (bindings.cpp, voxelGrid.cpp:166-178, 279-299):
      sparse grids with negative values, single voxels, full grids, and
      empty grids (make_tight raises);
and from its Python package, the 24 rotation matrices of the orientation
order (spectral_packer/rotations.py:41-89).
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]


def place_cases(rng):
    out = []
    for k in range(40):
        nx, ny, nz = (int(v) for v in rng.integers(3, 12, 3))
        ex, ey, ez = (int(v) for v in rng.integers(1, 7, 3))
        tray = np.zeros((nx, ny, nz), np.int32)
        mode = k % 4
        if mode >= 1:  # some occupied cells, ids up to 9, a few negative cells
            m = rng.random(tray.shape) < (0.08 if mode == 1 else 0.3)
            tray[m] = rng.integers(1, 10, int(m.sum()))
            tray[rng.random(tray.shape) < 0.03] = -2
        item = (rng.random((ex, ey, ez)) < 0.7).astype(np.int32) * rng.integers(1, 4, (ex, ey, ez)).astype(np.int32)
        item[rng.random(item.shape) < 0.05] = -1
        pos = tuple(int(v) for v in rng.integers(-3, np.array([nx, ny, nz]) + 2))
        out.append((item, tray, pos, int(rng.integers(1, 300))))
    return out


def grid_cases(rng):
    out = [np.zeros((3, 4, 5), np.int32), np.ones((2, 3, 4), np.int32)]
    g = np.zeros((6, 7, 8), np.int32)
    g[4, 1, 6] = 3
    out.append(g)
    for k in range(12):
        shape = tuple(int(v) for v in rng.integers(1, 10, 3))
        g = np.zeros(shape, np.int32)
        m = rng.random(shape) < 0.1
        g[m] = rng.integers(-2, 5, int(m.sum()))
        out.append(g)
    return out


def main(ref_dir: str) -> None:
    sys.path.insert(0, str(Path(ref_dir).resolve()))
    import spectral_packer._core as R  # the reference's module, built from its sources

    rng = np.random.default_rng(424242)
    rec = {}
    for k, (item, tray, pos, val) in enumerate(place_cases(rng)):
        rec[f"place/{k}/item"], rec[f"place/{k}/tray"] = item, tray
        rec[f"place/{k}/pos"], rec[f"place/{k}/val"] = np.asarray(pos, np.int32), np.int32(val)
        try:
            rec[f"place/{k}/out"] = np.asarray(R.place_in_tray(item, tray, pos, val), np.int32)
        except RuntimeError as e:
            rec[f"place/{k}/error"] = np.asarray(str(e))
    rec["place_count"] = np.int32(k + 1)
    for k, g in enumerate(grid_cases(rng)):
        rec[f"grid/{k}/in"] = g
        lo, hi = R.get_bounds(g)
        rec[f"grid/{k}/bounds"] = np.asarray([lo, hi], np.int64)
        try:
            rec[f"grid/{k}/tight"] = np.asarray(R.make_tight(g), np.int32)
        except ValueError:
            rec[f"grid/{k}/tight_error"] = np.int8(1)
    rec["grid_count"] = np.int32(k + 1)
    from spectral_packer import rotations as RR  # the reference's unmodified package next to the module
    rec["rotation_matrices_3x3"] = np.asarray(RR.ROTATION_MATRICES_3x3, np.float64)
    # packing statistics and the result summary (packer.py:145-162, 582-601)
    from spectral_packer.packer import BinPacker, PackingResult
    for k in range(8):
        shape = tuple(int(v) for v in rng.integers(2, 30, 3))
        tray = np.zeros(shape, np.int32)
        if k:
            m = rng.random(shape) < [0.0005, 0.01, 0.2, 0.6, 0.9, 1.0, 0.05][k - 1]
            tray[m] = rng.integers(1, 40, int(m.sum()))
            tray[rng.random(shape) < 0.02] *= -1
        bp = BinPacker(shape, voxel_resolution=int(rng.integers(16, 200)), num_orientations=[1, 4, 6, 24][k % 4])
        dens, total, bbox = bp._calculate_stats(tray)
        placed, failed = int(rng.integers(0, 50)), int(rng.integers(0, 50))
        res = PackingResult(tray=tray, num_placed=placed, num_failed=failed, density=dens, total_volume=total,
                            bounding_box=bbox)
        rec[f"stats/{k}/tray"] = tray
        rec[f"stats/{k}/args"] = np.asarray([bp.voxel_resolution, bp.num_orientations, placed, failed], np.int64)
        rec[f"stats/{k}/density"] = np.float64(dens)
        rec[f"stats/{k}/total"] = np.int64(total)
        rec[f"stats/{k}/bbox"] = np.asarray(bbox if bbox else [[-1, -1, -1], [-1, -1, -1]], np.int64)
        rec[f"stats/{k}/summary"] = np.asarray(res.summary())
        rec[f"stats/{k}/repr"] = np.asarray(repr(bp))
    rec["stats_count"] = np.int32(8)
    np.savez_compressed(ROOT / "tests" / "golden" / "ref_host.npz", **rec)
    n_err = sum(1 for key in rec if key.endswith("/error"))
    print(f"{int(rec['place_count'])} place_in_tray cases ({n_err} raise), {int(rec['grid_count'])} grids")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    main(sys.argv[1])
