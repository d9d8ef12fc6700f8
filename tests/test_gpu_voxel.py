"""GPU voxelizer against the reference's own voxelize_stl outputs
(tests/golden/ref_voxels.npz) and against its CPU oracle (bit-exact), through
the C ABI and through voxelize_stl on binary and ASCII STL files."""
import numpy as np
import pytest

from oracle import psb_voxel_oracle as V
from tests import golden_vox, meshes

pytestmark = pytest.mark.gpu


GOLDEN = golden_vox.load()

CASES = [("box", meshes.box(), 16), ("box", meshes.box(), 24), ("box", meshes.box(), 40),
         ("flat", meshes.box(hi=(2.0, 1.0, 0.3)), 32), ("tetra", meshes.tetra(), 32),
         ("sphere", meshes.icosphere(2), 32), ("torus", meshes.torus(), 48),
         ("shifted", meshes.icosphere(1) + np.float32(3.7), 20)]


@pytest.mark.parametrize("name,tris,res", CASES, ids=[f"{c[0]}-{c[2]}" for c in CASES])
def test_voxelize_matches_oracle(gpu_core, name, tris, res):
    from psacking_b200.voxelize import voxelize_mesh
    try:
        want = V.voxelize(tris, res)
    except RuntimeError:  # no occupied cell (the unit cube at 40: every face skipped)
        with pytest.raises(RuntimeError, match="occupied"):
            voxelize_mesh(tris, res)
        return
    got = voxelize_mesh(tris, res)
    assert got.dtype == np.int32
    assert got.shape == want.shape and np.array_equal(got, want), name


def test_voxelize_stl_files(gpu_core, tmp_path):
    import psacking_b200 as p
    from psacking_b200.voxelize import write_stl
    tris = meshes.torus(n=16, m=8)
    b = tmp_path / "t.stl"
    write_stl(b, tris)
    a = tmp_path / "t_ascii.stl"
    lines = ["solid t"]
    for t in tris:
        lines += ["facet normal 0 0 0", "outer loop"] + [f"vertex {v[0]!r} {v[1]!r} {v[2]!r}" for v in t.tolist()]
        lines += ["endloop", "endfacet"]
    a.write_text("\n".join(lines + ["endsolid t"]) + "\n")
    gb = p.voxelize_stl(str(b), 40)
    ga = p.voxelize_stl(str(a), 40)
    assert np.array_equal(gb, ga) and np.array_equal(gb, V.voxelize(tris, 40))
    assert np.array_equal(gpu_core.voxelize_stl(str(b), 40), gb)   # the drop-in module's export
    with pytest.raises(RuntimeError, match="Voxelization failed"):
        p.voxelize_stl(str(tmp_path / "missing.stl"), 32)


@pytest.mark.parametrize("case", GOLDEN, ids=[c[0] for c in GOLDEN])
def test_voxelize_stl_matches_reference(gpu_core, tmp_path, case):
    """voxelize_stl on the STL file of each fixture mesh equals the
    reference's own output, or raises where the reference raised."""
    import psacking_b200 as p
    from psacking_b200.voxelize import write_stl
    name, tris, res, want = case
    path = tmp_path / "mesh.stl"
    write_stl(path, tris)
    if want is None:
        with pytest.raises(RuntimeError, match="Voxelization failed"):
            p.voxelize_stl(str(path), res)
        return
    got = p.voxelize_stl(str(path), res)
    assert got.dtype == np.int32 and got.shape == want.shape and np.array_equal(got, want), name
