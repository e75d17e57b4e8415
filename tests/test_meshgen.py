"""The synthetic workload generators: sizes of the benchmark configurations, conforming meshes,
positive volumes and complete boundary markers."""
import numpy as np
import pytest

from euler3d_b200 import meshgen as mg
from euler3d_b200.solver import Mesh


def test_bump_channel_sizes():
    raw = mg.bump_channel()
    assert raw.n_cells == 64 * 32 * 2
    a = Mesh.from_raw(raw).arrays()
    assert (a["n_faces"], a["n_faces_int"]) == (14528, 10048)
    assert a["n_faces"] - a["n_faces_int"] == sum(m.vtk.size for m in raw.markers)


def test_biconvex_ogrid_small():
    raw = mg.biconvex_ogrid(32, 16, 2)
    assert raw.n_cells == 32 * 16 * 2 * 2
    a = Mesh.from_raw(raw).arrays()
    assert np.all(a["cell_volume"] > 0)
    assert a["n_faces"] - a["n_faces_int"] == a["wall_ghost"].size + a["farfield_ghost"].size + a["sym_ghost"].size
    # the O-grid closes on itself: no boundary faces besides wall, farfield and span planes
    assert a["wall_ghost"].size == 32 * 2 and a["farfield_ghost"].size == 32 * 2


@pytest.mark.parametrize("n", [2, 5])
def test_bump_box_tets_conforming(n):
    raw = mg.bump_box_tets(n)
    assert raw.n_cells == 6 * n ** 3
    a = Mesh.from_raw(raw).arrays()
    # every tetrahedron face is matched or on a marker
    assert a["n_faces"] - a["n_faces_int"] == 12 * n * n
    assert a["wall_ghost"].size + a["farfield_ghost"].size + a["sym_ghost"].size == 12 * n * n
    assert np.all(a["cell_volume"] > 0)
    assert abs(a["cell_volume"].sum() - 64.0) < 64.0 * 0.02  # [0,4]^3 minus the small bump


@pytest.mark.parametrize("n", [2, 4])
def test_bump_box_pyramids_conforming(n):
    raw = mg.bump_box_pyramids(n)
    split = sum((i + j + k) % 2 for i in range(n) for j in range(n) for k in range(n))
    assert raw.n_cells == n ** 3 - split + 6 * split
    assert set(np.unique(raw.elem_vtk)) == {mg.VTK_HEXA, mg.VTK_PYRAMID}
    a = Mesh.from_raw(raw).arrays()
    # every face is matched or on a marker: the box's 6 n^2 boundary quadrilaterals
    assert a["n_faces"] - a["n_faces_int"] == 6 * n * n
    assert a["wall_ghost"].size + a["farfield_ghost"].size + a["sym_ghost"].size == 6 * n * n
    assert np.all(a["cell_volume"] > 0)
    assert abs(a["cell_volume"].sum() - 64.0) < 64.0 * 0.02


def test_generators_are_seeded():
    a, b = mg.bump_channel(seed=3), mg.bump_channel(seed=3)
    assert np.array_equal(a.xyz, b.xyz)
    assert not np.array_equal(a.xyz, mg.bump_channel(seed=4).xyz)


def test_su2_roundtrip(tmp_path):
    raw = mg.biconvex_ogrid(12, 5, 2)
    p = tmp_path / "m.par"
    mg.write_su2(raw, str(p))
    x = Mesh.read(str(p)).arrays()
    y = Mesh.from_raw(raw).arrays()
    for k in ("face2cell", "face_normal", "cell_volume", "sym_face"):
        assert np.array_equal(x[k], y[k])
