// Host-side mesh preparation for the Euler3D solver path: face connectivity, geometric
// metrics and boundary ghost classification, in the reference's own cell/face numbering.
//
// The reference builds these once per partition before the solver loop
// (src/connectivity/Connectivity.cpp:70-262, src/mesh/Metrics.cpp:9-335,
// include/mesh/Mesh.hpp:471-707).  Its numbering conventions are reproduced exactly
// (faces numbered by first encounter over (element, local face), interior faces first,
// left cell < right cell, ghost of boundary face f = nElem + f - nFaceInt) with an
// O(N) bucket match instead of the reference's O(N * nNode) scan, so meshes of tens of
// millions of cells are prepared in seconds.  Metrics follow the reference's formulas in
// the same IEEE operation order, so the arrays are identical to the reference's.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace e3d {

struct RawMarker {
    std::string tag;
    std::vector<int32_t> vtk;        // surface VTK type per element (5 triangle, 9 quad, 8 pixel)
    std::vector<int32_t> node_ptr;   // CSR over elements
    std::vector<int32_t> nodes;
};

struct RawMesh {
    std::vector<double> xyz;         // 3 * n_nodes
    std::vector<int32_t> elem_vtk;   // 10 tetra, 12 hexa, 13 wedge, 14 pyramid
    std::vector<int32_t> elem_ptr;   // CSR over elements
    std::vector<int32_t> elem_nodes;
    std::vector<RawMarker> markers;
    int32_t n_nodes() const { return (int32_t)(xyz.size() / 3); }
    int32_t n_elems() const { return (int32_t)elem_vtk.size(); }
};

// Everything the solver path consumes, in the reference's numbering.
struct PreparedMesh {
    int32_t n_cells = 0, n_faces = 0, n_faces_int = 0, n_nodes = 0;
    std::vector<int32_t> face2cell;            // 2 * n_faces (left, right); right >= n_cells is a ghost
    std::vector<int32_t> cell2face_ptr, cell2face;   // element -> faces in local-face order
    std::vector<int32_t> cell2cell;            // element -> neighbour or ghost, same layout
    std::vector<int32_t> face2node_ptr, face2node;
    std::vector<double> face_normal, face_unit_normal, face_center, face_area;
    std::vector<double> cell_volume, cell_centroid;
    // ghost classification: parallel (ghost, interior, face) lists per boundary kind
    std::vector<int32_t> wall_ghost, wall_interior, wall_face;
    std::vector<int32_t> farfield_ghost, farfield_interior, farfield_face;
    std::vector<int32_t> sym_ghost, sym_interior, sym_face;
    // a mesh merged from partition files: cells of partition p are [ptr[p], ptr[p+1]) (empty otherwise)
    std::vector<int32_t> partition_cell_ptr;
};

// The inter-partition faces a .par file lists for one neighbouring partition (NINTERNAL_MARKER=,
// src/parser/MeshPartition.cpp:39-112, written by src/partition/SU2Writer.cpp:107-124): for each
// face this partition's element, the neighbour's element (its local id there), the face's VTK type
// and the face's nodes in this partition's local numbering.
struct PartitionInterface {
    int32_t other = -1;
    std::vector<int32_t> this_elem, other_elem, vtk, node_ptr{0}, nodes;
};

// Throws std::runtime_error with a message on malformed input.
void prepare_mesh(const RawMesh &raw, double cref, PreparedMesh &out, int n_threads = 0);

// SU2 / single-partition .par text reader (layout of src/parser/SU2MeshParser.cpp:32-240 and
// src/parser/MeshPartition.cpp:39-112).  A .par file's NINTERNAL_MARKER section must be empty
// (one domain); throws otherwise.
void read_su2(const std::string &path, RawMesh &out);

// One partition file of a multi-partition case, with its inter-partition faces.
void read_su2_partition(const std::string &path, RawMesh &out, std::vector<PartitionInterface> &interfaces);

// One mesh from the partitions of a case (the files E3D_PRE writes, src/partition/Partition.cpp):
// nodes duplicated across partitions are joined through the inter-partition faces both sides list
// in the same order with the nodes in the same order (src/partition/Partition.cpp:222-296);
// elements are concatenated partition by partition (cell_ptr[p] = first cell of partition p) and
// boundary markers merged by tag.  Throws on inconsistent partitions.
void merge_partitions(const std::vector<RawMesh> &parts, const std::vector<std::vector<PartitionInterface>> &ifc,
                      RawMesh &out, std::vector<int32_t> &cell_ptr);

}  // namespace e3d
