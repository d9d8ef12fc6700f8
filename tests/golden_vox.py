"""Reader of tests/golden/ref_voxels.npz: the reference's own voxelize_stl
outputs on seeded meshes (tests/golden/make_voxel_golden.py)."""
from pathlib import Path

import numpy as np

PATH = Path(__file__).resolve().parent / "golden" / "ref_voxels.npz"


def load():
    """[(name, triangles float32 [n,3,3], resolution, grid int32 or None when the reference raised)]."""
    z = np.load(PATH)
    out = []
    for name in z["names"].tolist():
        tris = z[f"{name}/tris"]
        res = int(z[f"{name}/res"])
        if f"{name}/error" in z.files:
            out.append((name, tris, res, None))
            continue
        shape = tuple(int(s) for s in z[f"{name}/shape"])
        n = int(np.prod(shape))
        g = np.unpackbits(z[f"{name}/bits"])[:n].reshape(shape).astype(np.int32)
        out.append((name, tris, res, g))
    return out


def load_save_vox():
    """[(grid int32, sha256 hex, byte count)] of the reference's save_vox files."""
    z = np.load(PATH)
    return [(z[f"savevox/{k}/grid"], str(z[f"savevox/{k}/sha256"]), int(z[f"savevox/{k}/nbytes"]))
            for k in range(int(z["savevox_count"]))]
