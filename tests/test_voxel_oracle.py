"""CPU checks of the voxelizer oracle: bit for bit against the reference's
own voxelize_stl outputs (tests/golden/ref_voxels.npz), and on meshes whose
voxelization is known by hand."""
import numpy as np
import pytest

from oracle import psb_voxel_oracle as V
from tests import golden_vox, meshes

GOLDEN = golden_vox.load()


@pytest.mark.parametrize("case", GOLDEN, ids=[c[0] for c in GOLDEN])
def test_oracle_matches_reference_voxelizer(case):
    name, tris, res, want = case
    if want is None:  # the reference found no occupied cell and raised
        with pytest.raises(RuntimeError):
            V.voxelize(tris, res)
        return
    got = V.voxelize(tris, res)
    assert got.shape == want.shape and np.array_equal(got, want), name


def test_golden_covers_the_wrapped_degeneracy_test():
    """The fixture holds cubes whose faces the reference skips (its 32-bit
    determinant wraps to zero when 0.95 * res is an integer) and cubes it
    rasterizes, so both sides of that test are pinned."""
    cubes = {c[2]: c[3] for c in GOLDEN if c[0].startswith("cube-")}
    assert cubes[20] is None and cubes[40] is None and cubes[60] is None
    assert cubes[16] is not None and cubes[44] is not None


def test_merge_is_rank_of_position():
    tris = meshes.box()
    pos, idx = V.merge_vertices_exact(tris)
    assert len(pos) == 8
    assert all(tuple(pos[i]) < tuple(pos[i + 1]) for i in range(7))
    assert np.array_equal(pos[idx], tris)


def expected_cube(res):
    """The cube spans [0.025, 0.975] * res along every axis (5 % margin).  A
    face marks the pixels whose centre (i + 0.5) lies inside that span, in
    the voxel layer floor(face coordinate); a voxel is set by a face in one
    axis view (edge pixels of one face are not covered by the others)."""
    lo, hi = 0.025 * res, 0.975 * res
    cov = [i for i in range(res) if lo <= i + 0.5 <= hi]
    a, b = min(cov), max(cov)
    layers = (int(np.floor(lo)), int(np.floor(hi)))
    g = np.zeros((res, res, res), np.int32)
    for L in layers:
        g[a:b + 1, a:b + 1, L] = 1
        g[L, a:b + 1, a:b + 1] = 1
        g[a:b + 1, L, a:b + 1] = 1
    return V.make_tight(g)


def test_cube_faces():
    for res in (8, 16, 24, 44):
        g = V.voxelize(meshes.box(), res)
        assert np.array_equal(g, expected_cube(res)), res
    # below a 1/2-voxel margin every face covers the whole side: a full shell
    g = V.voxelize(meshes.box(), 16)
    shell = np.ones((16, 16, 16), np.int32)
    shell[1:-1, 1:-1, 1:-1] = 0
    assert np.array_equal(g, shell)


def test_flat_box_aspect():
    g = V.voxelize(meshes.box(hi=(2.0, 1.0, 0.5)), 16)
    assert g.shape == (16, 8, 4)


def test_closed_surfaces_have_no_holes_along_axes():
    """For a closed surface every axis line through the solid meets it an
    even number of times: a column of the shell never has a single voxel
    gap between two occupied runs that a watertight raster would fill."""
    g = V.voxelize(meshes.icosphere(1), 16)
    assert g.sum() > 0
    c = np.array(g.shape) // 2
    assert g[:, c[1], c[2]].sum() >= 2 and g[c[0], :, c[2]].sum() >= 2 and g[c[0], c[1], :].sum() >= 2


def test_stl_reader_binary_and_ascii(tmp_path):
    from psacking_b200.voxelize import read_stl, write_stl
    tris = meshes.tetra()
    write_stl(tmp_path / "a.stl", tris)
    assert np.array_equal(read_stl(tmp_path / "a.stl"), tris)
    txt = ["solid x"]
    for t in tris:
        txt += ["facet normal 0 0 1", "outer loop"] + [f"vertex {v[0]!r} {v[1]!r} {v[2]!r}" for v in t.tolist()]
        txt += ["endloop", "endfacet"]
    (tmp_path / "b.stl").write_text("\n".join(txt + ["endsolid x"]))
    assert np.array_equal(read_stl(tmp_path / "b.stl"), tris)
