"""The product's mesh preparation (connectivity, metrics, ghost lists) against the reference.

Bit for bit against the arrays the reference itself produced (golden fixtures), and against the
known answers of the reference's own unit tests.
"""
import os

import numpy as np
import pytest

from euler3d_b200 import _lib
from euler3d_b200 import meshgen as mg
from euler3d_b200.solver import Mesh

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
ARRAYS = ("face2cell", "cell2face_ptr", "cell2face", "cell2cell", "face2node_ptr", "face2node", "face_normal",
          "face_unit_normal", "face_center", "face_area", "cell_volume", "cell_centroid", "wall_ghost",
          "wall_interior", "wall_face", "farfield_ghost", "farfield_interior", "farfield_face", "sym_ghost",
          "sym_interior", "sym_face")


def raw_from_fixture(z):
    markers, off = [], 0
    for tag, n in zip(z["raw_marker_tags"], z["raw_marker_sizes"]):
        nodes = z["raw_marker_nodes"][off:off + n]
        off += n
        vtk = np.where(nodes[:, 3] < 0, mg.VTK_TRIANGLE, mg.VTK_QUAD).astype(np.int32)
        markers.append(mg.Marker(str(tag), vtk, nodes))
    ptr, nodes = z["raw_elem_ptr"], z["raw_elem_nodes"]
    packed = np.full((len(z["raw_elem_vtk"]), 8), -1, np.int32)
    for i in range(len(ptr) - 1):
        packed[i, : ptr[i + 1] - ptr[i]] = nodes[ptr[i]:ptr[i + 1]]
    return mg.RawMesh(z["raw_xyz"], z["raw_elem_vtk"], packed, markers)


@pytest.mark.parametrize("name", ["channel", "channel_supersonic", "ogrid", "tets", "pyramids"])
def test_prepared_arrays_equal_reference(name):
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    ours = Mesh.from_raw(raw_from_fixture(z)).arrays()
    for k in ("n_cells", "n_faces", "n_faces_int"):
        assert ours[k] == int(z[f"mesh_{k}"])
    for k in ARRAYS:
        assert np.array_equal(ours[k], z[f"mesh_{k}"]), k


def reference_mesh(tmp_path, key):
    z = np.load(os.path.join(GOLDEN, "reference_test_meshes.npz"))
    par = tmp_path / f"{key}.par"
    par.write_bytes(z[f"{key}__par"].tobytes())
    return Mesh.read(str(par)), z


@pytest.mark.parametrize("key", ["StructuredBlock_8", "naca0012_9x9x5_unittest_mesh", "stackedCubes",
                                 "stackedTetrahedron"])
def test_reference_test_meshes(tmp_path, key):
    mesh, z = reference_mesh(tmp_path, key)
    ours = mesh.arrays()
    for k in ARRAYS:
        assert np.array_equal(ours[k], z[f"{key}__{k}"]), k


def test_connectivity_known_answers(tmp_path):
    """Expected values of the reference's test/Test_Connectivity.cpp:17-128 on StructuredBlock_8."""
    mesh, _ = reference_mesh(tmp_path, "StructuredBlock_8")
    a = mesh.arrays()
    assert a["n_faces"] == 36
    ptr = a["cell2face_ptr"]
    e2e = lambda e: list(a["cell2cell"][ptr[e]:ptr[e + 1]])  # noqa: E731
    e2f = lambda e: list(a["cell2face"][ptr[e]:ptr[e + 1]])  # noqa: E731
    assert e2e(0) == [8, 9, 1, 2, 10, 4]
    assert e2e(3) == [17, 1, 18, 19, 2, 7]
    assert e2e(7) == [3, 5, 29, 30, 6, 31]
    assert e2f(0) == [12, 13, 0, 1, 14, 2]
    assert e2f(3) == [21, 3, 22, 23, 5, 7]
    assert e2f(7) == [7, 10, 33, 34, 11, 35]
    f2c = a["face2cell"].reshape(-1, 2)
    assert list(f2c[0]) == [0, 1] and list(f2c[29]) == [5, 25] and list(f2c[35]) == [7, 31]
    fp = a["face2node_ptr"]
    f2n = lambda f: list(a["face2node"][fp[f]:fp[f + 1]])  # noqa: E731
    assert f2n(0) == [1, 4, 13, 10]
    assert f2n(29) == [19, 20, 23, 22]
    assert f2n(35) == [22, 23, 26, 25]


def test_metric_known_answers():
    """Two stacked unit hexes: volume 0.125 and centroids of test/Test_Parser.cpp:215-225."""
    xyz = np.array([[x, y, z] for z in (0.0, 0.5, 1.0) for y in (0.0, 0.5) for x in (0.0, 0.5)])
    hexes = np.array([[0, 1, 3, 2, 4, 5, 7, 6], [4, 5, 7, 6, 8, 9, 11, 10]], np.int32)
    faces = []
    for h in hexes:
        for q in ([0, 3, 2, 1], [0, 1, 5, 4], [1, 2, 6, 5], [2, 3, 7, 6], [3, 0, 4, 7], [4, 5, 6, 7]):
            faces.append(tuple(sorted(h[q])))
    bnd = [f for f in set(faces) if faces.count(f) == 1]
    raw = mg.RawMesh(xyz, np.full(2, mg.VTK_HEXA, np.int32), hexes,
                     [mg.Marker("farfield", np.full(len(bnd), mg.VTK_QUAD, np.int32), np.array(bnd, np.int32))])
    a = Mesh.from_raw(raw).arrays()
    assert np.allclose(a["cell_volume"], 0.125, rtol=1e-14)
    assert np.allclose(a["cell_centroid"].reshape(-1, 3), [[0.25, 0.25, 0.25], [0.25, 0.25, 0.75]])
    assert np.allclose(a["face_area"], 0.25)


def test_bc_classification_counts():
    a = Mesh.from_raw(mg.bump_channel()).arrays()
    assert a["n_cells"] == 4096 and a["n_faces"] == 14528 and a["n_faces_int"] == 10048
    assert a["wall_ghost"].size == 128 and a["farfield_ghost"].size == 128 and a["sym_ghost"].size == 4224


def test_malformed_mesh_is_rejected(tmp_path):
    bad = tmp_path / "bad.su2"
    bad.write_text("NDIME= 3\nNELEM= 1\n11 0 1 2 3 4 5 6 7\n")
    with pytest.raises(_lib.E3DError) as e:
        Mesh.read(str(bad))
    assert e.value.status == _lib.E3D_ERR_MESH and "VTK" in str(e.value)
    with pytest.raises(_lib.E3DError) as e:
        Mesh.read(str(tmp_path / "missing.su2"))
    assert e.value.status == _lib.E3D_ERR_MESH
    raw = mg.bump_channel(4, 3, 2)
    raw.elem_nodes[0, 1] = raw.xyz.shape[0] + 5  # node out of range
    with pytest.raises(_lib.E3DError):
        Mesh.from_raw(raw)
