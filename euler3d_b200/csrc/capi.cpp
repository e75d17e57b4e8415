// Mesh half of the C ABI (include/euler3d_b200.h) plus status strings and error reporting.
#include <cstdio>
#include <cstring>
#include <memory>
#include <new>
#include <string>

#include "common.hpp"
#include "euler3d_b200.h"
#include "mesh_prep.hpp"

namespace e3d {

namespace {
thread_local std::string g_last_error;
}

void set_last_error(const std::string &msg) { g_last_error = msg; }

}  // namespace e3d

using namespace e3d;

struct e3d_mesh {
    PreparedMesh m;
};

extern "C" {

const char *e3d_last_error(void) { return g_last_error.c_str(); }

int32_t e3d_abi_version(void) { return E3D_ABI_VERSION; }

const char *e3d_status_string(e3d_status s) {
    switch (s) {
        case E3D_OK: return "ok";
        case E3D_ERR_INVALID_ARG: return "invalid argument";
        case E3D_ERR_OOM: return "out of memory";
        case E3D_ERR_NONFINITE: return "non-finite solution";
        case E3D_ERR_TIMEOUT: return "timeout";
        case E3D_ERR_CUDA: return "CUDA error";
        case E3D_ERR_MESH: return "mesh error";
    }
    return "unknown status";
}

e3d_status e3d_mesh_read(const char *path, double cref, int32_t n_threads, e3d_mesh **out) {
    if (!path || !out) {
        set_last_error("NULL argument");
        return E3D_ERR_INVALID_ARG;
    }
    *out = nullptr;
    std::unique_ptr<e3d_mesh> mesh(new (std::nothrow) e3d_mesh());
    if (!mesh) return E3D_ERR_OOM;
    e3d_status st = guarded([&] {
        if (!(cref != 0.0)) throw Error(E3D_ERR_INVALID_ARG, "cref must be non-zero");
        RawMesh raw;
        read_su2(path, raw);
        prepare_mesh(raw, cref, mesh->m, n_threads);
    });
    if (st == E3D_OK) *out = mesh.release();
    return st;
}

e3d_status e3d_mesh_read_partitions(const char *const *paths, int32_t n_parts, double cref, int32_t n_threads,
                                    e3d_mesh **out) {
    if (!paths || !out || n_parts <= 0) {
        set_last_error("NULL argument or no partition files");
        return E3D_ERR_INVALID_ARG;
    }
    *out = nullptr;
    std::unique_ptr<e3d_mesh> mesh(new (std::nothrow) e3d_mesh());
    if (!mesh) return E3D_ERR_OOM;
    e3d_status st = guarded([&] {
        if (!(cref != 0.0)) throw Error(E3D_ERR_INVALID_ARG, "cref must be non-zero");
        std::vector<RawMesh> parts(n_parts);
        std::vector<std::vector<PartitionInterface>> ifc(n_parts);
        for (int p = 0; p < n_parts; p++) {
            if (!paths[p]) throw Error(E3D_ERR_INVALID_ARG, "partition path is NULL");
            read_su2_partition(paths[p], parts[p], ifc[p]);
        }
        RawMesh merged;
        std::vector<int32_t> cell_ptr;
        merge_partitions(parts, ifc, merged, cell_ptr);
        parts.clear();
        prepare_mesh(merged, cref, mesh->m, n_threads);
        mesh->m.partition_cell_ptr = std::move(cell_ptr);
    });
    if (st == E3D_OK) *out = mesh.release();
    return st;
}

e3d_status e3d_mesh_from_arrays(int32_t n_nodes, const double *xyz, int32_t n_elems, const int32_t *elem_vtk,
                                const int32_t *elem_ptr, const int32_t *elem_nodes, int32_t n_markers,
                                const char *const *marker_tags, const int32_t *marker_ptr, const int32_t *face_ptr,
                                const int32_t *face_nodes, double cref, int32_t n_threads, e3d_mesh **out) {
    if (!out) {
        set_last_error("NULL output pointer");
        return E3D_ERR_INVALID_ARG;
    }
    *out = nullptr;
    std::unique_ptr<e3d_mesh> mesh(new (std::nothrow) e3d_mesh());
    if (!mesh) return E3D_ERR_OOM;
    e3d_status st = guarded([&] {
        if (n_nodes <= 0 || n_elems <= 0 || n_markers < 0 || !xyz || !elem_vtk || !elem_ptr || !elem_nodes)
            throw Error(E3D_ERR_INVALID_ARG, "invalid volume mesh arrays");
        if (n_markers > 0 && (!marker_tags || !marker_ptr || !face_ptr || !face_nodes))
            throw Error(E3D_ERR_INVALID_ARG, "invalid marker arrays");
        if (!(cref != 0.0)) throw Error(E3D_ERR_INVALID_ARG, "cref must be non-zero");
        RawMesh raw;
        raw.xyz.assign(xyz, xyz + 3 * (size_t)n_nodes);
        raw.elem_vtk.assign(elem_vtk, elem_vtk + n_elems);
        raw.elem_ptr.assign(elem_ptr, elem_ptr + n_elems + 1);
        if (raw.elem_ptr[0] != 0) throw Error(E3D_ERR_INVALID_ARG, "elem_ptr[0] must be 0");
        raw.elem_nodes.assign(elem_nodes, elem_nodes + elem_ptr[n_elems]);
        for (int32_t m = 0; m < n_markers; m++) {
            RawMarker mk;
            if (!marker_tags[m]) throw Error(E3D_ERR_INVALID_ARG, "marker tag is NULL");
            mk.tag = marker_tags[m];
            int32_t f0 = marker_ptr[m], f1 = marker_ptr[m + 1];
            if (f1 < f0) throw Error(E3D_ERR_INVALID_ARG, "marker_ptr decreasing");
            mk.node_ptr.push_back(0);
            for (int32_t f = f0; f < f1; f++) {
                int32_t n0 = face_ptr[f], n1 = face_ptr[f + 1];
                if (n1 - n0 != 3 && n1 - n0 != 4) throw Error(E3D_ERR_INVALID_ARG, "marker face must have 3 or 4 nodes");
                mk.vtk.push_back(n1 - n0 == 3 ? 5 : 9);
                mk.nodes.insert(mk.nodes.end(), face_nodes + n0, face_nodes + n1);
                mk.node_ptr.push_back((int32_t)mk.nodes.size());
            }
            raw.markers.push_back(std::move(mk));
        }
        prepare_mesh(raw, cref, mesh->m, n_threads);
    });
    if (st == E3D_OK) *out = mesh.release();
    return st;
}

e3d_status e3d_mesh_info_get(const e3d_mesh *mesh, e3d_mesh_info *info) {
    if (!mesh || !info) {
        set_last_error("NULL argument");
        return E3D_ERR_INVALID_ARG;
    }
    const PreparedMesh &m = mesh->m;
    info->n_cells = m.n_cells;
    info->n_faces = m.n_faces;
    info->n_faces_int = m.n_faces_int;
    info->n_nodes = m.n_nodes;
    info->n_wall = (int32_t)m.wall_ghost.size();
    info->n_farfield = (int32_t)m.farfield_ghost.size();
    info->n_sym = (int32_t)m.sym_ghost.size();
    return E3D_OK;
}

e3d_status e3d_mesh_array(const e3d_mesh *mesh, const char *name, const void **data, int64_t *count,
                          int32_t *is_double) {
    if (!mesh || !name || !data || !count || !is_double) {
        set_last_error("NULL argument");
        return E3D_ERR_INVALID_ARG;
    }
    const PreparedMesh &m = mesh->m;
    struct I {
        const char *n;
        const std::vector<int32_t> *v;
    };
    struct D {
        const char *n;
        const std::vector<double> *v;
    };
    const I ints[] = {{"face2cell", &m.face2cell},         {"cell2face_ptr", &m.cell2face_ptr},
                      {"cell2face", &m.cell2face},         {"cell2cell", &m.cell2cell},
                      {"face2node_ptr", &m.face2node_ptr}, {"face2node", &m.face2node},
                      {"partition_cell_ptr", &m.partition_cell_ptr},
                      {"wall_ghost", &m.wall_ghost},       {"wall_interior", &m.wall_interior},
                      {"wall_face", &m.wall_face},         {"farfield_ghost", &m.farfield_ghost},
                      {"farfield_interior", &m.farfield_interior}, {"farfield_face", &m.farfield_face},
                      {"sym_ghost", &m.sym_ghost},         {"sym_interior", &m.sym_interior},
                      {"sym_face", &m.sym_face}};
    const D dbls[] = {{"face_normal", &m.face_normal}, {"face_unit_normal", &m.face_unit_normal},
                      {"face_center", &m.face_center}, {"face_area", &m.face_area},
                      {"cell_volume", &m.cell_volume}, {"cell_centroid", &m.cell_centroid}};
    for (const I &e : ints)
        if (!std::strcmp(e.n, name)) {
            *data = e.v->data();
            *count = (int64_t)e.v->size();
            *is_double = 0;
            return E3D_OK;
        }
    for (const D &e : dbls)
        if (!std::strcmp(e.n, name)) {
            *data = e.v->data();
            *count = (int64_t)e.v->size();
            *is_double = 1;
            return E3D_OK;
        }
    set_last_error(std::string("unknown mesh array '") + name + "'");
    return E3D_ERR_INVALID_ARG;
}

e3d_status e3d_mesh_write_boundary(const e3d_mesh *mesh, const char *path) {
    return guarded([&] {
        if (!mesh || !path) throw Error(E3D_ERR_INVALID_ARG, "NULL argument");
        const PreparedMesh &m = mesh->m;
        FILE *f = std::fopen(path, "w");
        if (!f) throw Error(E3D_ERR_INVALID_ARG, std::string("cannot open ") + path + " for writing");
        std::fprintf(f, "NOMBRE DE CELLULES= %zu\n", m.wall_ghost.size());
        for (size_t i = 0; i < m.wall_ghost.size(); i++) {
            const int face = m.wall_face[i];
            const int a = m.face2node_ptr[face], b = m.face2node_ptr[face + 1];
            std::fprintf(f, "%9d%9d", m.wall_interior[i], b - a);
            for (int k = a; k < b; k++) std::fprintf(f, "%9d", m.face2node[k]);
            std::fprintf(f, "\n");
        }
        if (std::fclose(f) != 0) throw Error(E3D_ERR_INVALID_ARG, "writing the boundary file failed");
    });
}

e3d_status e3d_mesh_describe(const e3d_mesh *mesh, e3d_mesh_desc *d) {
    if (!mesh || !d) {
        set_last_error("NULL argument");
        return E3D_ERR_INVALID_ARG;
    }
    const PreparedMesh &m = mesh->m;
    std::memset(d, 0, sizeof *d);
    d->n_cells = m.n_cells;
    d->n_faces = m.n_faces;
    d->n_faces_int = m.n_faces_int;
    d->face2cell = m.face2cell.data();
    d->face_unit_normal = m.face_unit_normal.data();
    d->face_normal = m.face_normal.data();
    d->face_area = m.face_area.data();
    d->face_center = m.face_center.data();
    d->cell_volume = m.cell_volume.data();
    d->cell2face_ptr = m.cell2face_ptr.data();
    d->cell2face = m.cell2face.data();
    d->n_wall = (int32_t)m.wall_ghost.size();
    d->wall_ghost = m.wall_ghost.data();
    d->wall_interior = m.wall_interior.data();
    d->wall_face = m.wall_face.data();
    d->n_farfield = (int32_t)m.farfield_ghost.size();
    d->farfield_ghost = m.farfield_ghost.data();
    d->farfield_interior = m.farfield_interior.data();
    d->farfield_face = m.farfield_face.data();
    d->n_sym = (int32_t)m.sym_ghost.size();
    d->sym_ghost = m.sym_ghost.data();
    d->sym_interior = m.sym_interior.data();
    d->sym_face = m.sym_face.data();
    return E3D_OK;
}

void e3d_mesh_destroy(e3d_mesh *mesh) { delete mesh; }

}  // extern "C"
