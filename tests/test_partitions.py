"""Multi-partition cases (PARTITION_FILES= n): the partition files are merged into one mesh for one
GPU.  The merged mesh must be the mesh the partitions were cut from -- the same cells (bit-identical
volumes), faces and boundary faces -- checked on the reference's own partitioned test case and on
partitions of the benchmark families written in the reference's layout.

Its cells are numbered partition by partition, so its faces are numbered differently from the uncut
mesh's, and two parts of the reference's discretization follow the numbering: Harten's entropy fix
takes delta from the sound speed of a face's left (lower-numbered) cell
(src/solver/ConvectiveFluxesSchemes.cpp:63-77), and the unit normal of a non-planar quad depends on
which node starts the face (src/mesh/Metrics.cpp:116-140).  On the uniform-flow reference block the
two runs agree to round-off; on the jittered benchmark meshes to about 1e-6 after 15 iterations."""
import os

import numpy as np
import pytest

import pyoracle as po
from euler3d_b200 import _lib
from euler3d_b200 import meshgen as mg
from euler3d_b200.solver import Mesh

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def match(merged, orig):
    """perm[i] = the original cell that merged cell i is (nearest cell centroid; the centroids of a
    cell agree to round-off whatever the face numbering)."""
    from scipy.spatial import cKDTree

    cm, co = merged["cell_centroid"].reshape(-1, 3), orig["cell_centroid"].reshape(-1, 3)
    dist, perm = cKDTree(co).query(cm)
    assert np.max(dist) < 1e-12
    assert np.array_equal(np.sort(perm), np.arange(orig["n_cells"]))
    return perm


def same_mesh(merged, orig):
    perm = match(merged, orig)
    assert (merged["n_faces"], merged["n_faces_int"]) == (orig["n_faces"], orig["n_faces_int"])
    assert np.array_equal(merged["cell_volume"], orig["cell_volume"][perm])
    for kind in ("wall", "farfield", "sym"):
        assert merged[f"{kind}_ghost"].size == orig[f"{kind}_ghost"].size, kind
    return perm


def same_flow(merged, orig, perm, iters=15, rtol=1e-12):
    fl = po.flow(0.6, 1.0, 1.4, 1.2)
    res = []
    for a in (merged, orig):
        m = po.Mesh(a)
        s = po.freestream(m, fl)
        _, h = po.run(m, fl, s, iters)
        res.append((s.a, h))
    (sm, hm), (so, ho) = res
    n = merged["n_cells"]
    for k in ("rho", "u", "p", "E"):
        ref = so[k][:n][perm]
        assert np.max(np.abs(sm[k][:n] - ref) / np.maximum(np.abs(ref), 1e-3)) < rtol, k
    assert np.all(np.abs(hm - ho) <= rtol * np.abs(ho) + 1e-15)  # round-off-level RMS on uniform flow


def reference_case(tmp_path):
    z = np.load(os.path.join(GOLDEN, "reference_partitions.npz"))
    paths = []
    for i in range(4):
        p = tmp_path / f"StructuredBlock_8_p{i}.par"
        p.write_bytes(z[f"StructuredBlock_8_p{i}_par"].tobytes())
        paths.append(str(p))
    su2 = tmp_path / "StructuredBlock_8.par"
    su2.write_bytes(z["StructuredBlock_8_su2"].tobytes().rstrip(b"\n") + b"\nNINTERNAL_MARKER= 0\n")
    return paths, str(su2)


def test_reference_partitions_merge_to_their_mesh(tmp_path):
    paths, whole = reference_case(tmp_path)
    m = Mesh.read_partitions(paths)
    merged, orig = m.arrays(), Mesh.read(whole).arrays()
    assert merged["n_cells"] == orig["n_cells"] == 8
    assert np.array_equal(m.partition_cell_ptr(), [0, 2, 4, 6, 8])
    perm = same_mesh(merged, orig)
    same_flow(merged, orig, perm)


@pytest.mark.parametrize("family,parts", [("channel", 3), ("tets", 4), ("ogrid", 5)])
def test_written_partitions_round_trip(family, parts, tmp_path):
    raw = {"channel": lambda: mg.bump_channel(16, 8, 2), "tets": lambda: mg.bump_box_tets(5),
           "ogrid": lambda: mg.biconvex_ogrid(24, 12, 2)}[family]()
    paths = mg.write_partitions(raw, parts, str(tmp_path / "p#.par"))
    assert len(paths) == parts
    m = Mesh.read_partitions(paths)
    merged, orig = m.arrays(), Mesh.from_raw(raw).arrays()
    ptr = m.partition_cell_ptr()
    assert ptr.size == parts + 1 and ptr[-1] == orig["n_cells"]
    perm = same_mesh(merged, orig)
    same_flow(merged, orig, perm, rtol=1e-5)


def test_single_partition_file(tmp_path):
    raw = mg.bump_channel(8, 4, 2)
    p = str(tmp_path / "one.par")
    mg.write_su2(raw, p)
    a, b = Mesh.read_partitions([p]).arrays(), Mesh.read(p).arrays()
    for k in ("face2cell", "cell_volume", "face_normal"):
        assert np.array_equal(a[k], b[k])


def test_inconsistent_partitions_are_refused(tmp_path):
    raw = mg.bump_channel(16, 8, 2)
    paths = mg.write_partitions(raw, 3, str(tmp_path / "p#.par"))
    with pytest.raises(_lib.E3DError) as e:
        Mesh.read_partitions(paths[:2])  # partition 2 missing
    assert e.value.status == _lib.E3D_ERR_MESH
    # a partition file on its own is not a whole mesh
    with pytest.raises(_lib.E3DError):
        Mesh.read(paths[0])
    # corrupt one shared face's node list
    txt = open(paths[1]).read().splitlines()
    i = max(k for k, line in enumerate(txt) if line.startswith("NELEM_MPI="))
    row = txt[i + 1].split()
    row[3], row[4] = row[4], row[3]
    txt[i + 1] = " ".join(row)
    open(paths[1], "w").write("\n".join(txt) + "\n")
    with pytest.raises(_lib.E3DError):
        Mesh.read_partitions(paths)
