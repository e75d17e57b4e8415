// Host-side mesh preparation: connectivity, metrics and ghost classification in the
// reference's numbering.  See mesh_prep.hpp for the contract.
#include "mesh_prep.hpp"

#include <algorithm>
#include <array>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cstdint>
#include <fstream>
#include <numeric>
#include <stdexcept>
#include <string>
#include <thread>
#include <unordered_map>

namespace e3d {
namespace {

// Local faces of each volume element, as local node indices in the order the face's node
// list is stored (reference tables: include/connectivity/Connectivity.hpp:36-44; VTK
// ordering).  The face order and node order fix the reference's face numbering, face2node
// lists and therefore the sign of every face normal, so they are reproduced as they are.
struct ElemType {
    int vtk, n_nodes, n_faces;
    int face_nodes[6];        // nodes per face
    int face_local[6][4];     // local node indices
};
constexpr ElemType kTetra{10, 4, 4, {3, 3, 3, 3}, {{0, 2, 1}, {0, 1, 3}, {1, 2, 3}, {2, 0, 3}}};
constexpr ElemType kHexa{12, 8, 6, {4, 4, 4, 4, 4, 4},
                         {{0, 3, 2, 1}, {0, 1, 5, 4}, {1, 2, 6, 5}, {2, 3, 7, 6}, {3, 0, 4, 7}, {4, 5, 6, 7}}};
constexpr ElemType kWedge{13, 6, 5, {3, 4, 4, 4, 3}, {{0, 1, 2}, {0, 2, 5, 3}, {0, 3, 4, 1}, {1, 4, 5, 2}, {3, 5, 4}}};
constexpr ElemType kPyramid{14, 5, 5, {4, 3, 3, 3, 3}, {{0, 3, 2, 1}, {0, 1, 4}, {1, 2, 4}, {2, 3, 4}, {3, 0, 4}}};

const ElemType *elem_type(int vtk) {
    switch (vtk) {
        case 10: return &kTetra;
        case 12: return &kHexa;
        case 13: return &kWedge;
        case 14: return &kPyramid;
        default: return nullptr;
    }
}

using Key = std::array<int32_t, 4>;  // sorted node ids, -1 padding for triangles

inline Key make_key(const int32_t *nodes, int n) {
    Key k{nodes[0], nodes[1], nodes[2], n == 4 ? nodes[3] : -1};
    if (n == 3) {
        std::sort(k.begin(), k.begin() + 3);
    } else {
        std::sort(k.begin(), k.end());
    }
    return k;
}

// Smallest node of a key (triangles carry -1 in the last slot).
inline int32_t key_min(const Key &k) { return k[0]; }

struct KeyHash {
    size_t operator()(const Key &k) const {
        uint64_t h = 1469598103934665603ull;
        for (int32_t v : k) {
            h ^= (uint32_t)v;
            h *= 1099511628211ull;
        }
        return (size_t)h;
    }
};

int pick_threads(int requested) {
    if (requested > 0) return requested;
    unsigned hc = std::thread::hardware_concurrency();
    return hc ? (int)std::min(hc, 64u) : 1;
}

template <typename F>
void parallel_for(int64_t n, int threads, F &&fn) {
    if (threads <= 1 || n < 4096) {
        fn((int64_t)0, n);
        return;
    }
    std::vector<std::thread> pool;
    int64_t chunk = (n + threads - 1) / threads;
    for (int t = 0; t < threads; t++) {
        int64_t b = t * chunk, e = std::min(n, b + chunk);
        if (b >= e) break;
        pool.emplace_back([&fn, b, e] { fn(b, e); });
    }
    for (auto &th : pool) th.join();
}

// --- small vector helpers written in the reference's operation order (Vector3, include/utils/Vector3.h)
struct V3 {
    double x, y, z;
};
inline V3 sub(const V3 &a, const V3 &b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 add(const V3 &a, const V3 &b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 mul(const V3 &a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 divs(const V3 &a, double s) { return {a.x / s, a.y / s, a.z / s}; }
inline V3 cross(const V3 &a, const V3 &b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline double dot(const V3 &a, const V3 &b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double length(const V3 &a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
// half the cross product's length (computeTriangleArea, src/mesh/Metrics.cpp:60-62)
inline double tri_area(const V3 &a, const V3 &b) { return length(mul(cross(a, b), 0.5)); }

// Tetrahedron volume from its six edge lengths (Metrics::TetrahedronVolume,
// src/mesh/Metrics.cpp:311-331).  The squared lengths are squares of the rounded lengths,
// as there, so the result matches the reference's bits.
double tet_volume(const V3 &p0, const V3 &p1, const V3 &p2, const V3 &p3) {
    double U = length(sub(p0, p1)), V = length(sub(p1, p2)), W = length(sub(p2, p0));
    double u = length(sub(p2, p3)), v = length(sub(p0, p3)), w = length(sub(p3, p1));
    double u2 = u * u, v2 = v * v, w2 = w * w, U2 = U * U, V2 = V * V, W2 = W * W;
    double X = v2 + w2 - U2, Y = w2 + u2 - V2, Z = u2 + v2 - W2;
    double a = 4 * (u2 * v2 * w2) - u2 * (X * X) - v2 * (Y * Y) - w2 * (Z * Z) + X * Y * Z;
    double vol = std::sqrt(a);
    vol /= 12.0;
    return vol;
}
inline V3 tet_centroid(const V3 &a, const V3 &b, const V3 &c, const V3 &d) {
    return divs(add(add(add(a, b), c), d), 4.0);
}

}  // namespace

void prepare_mesh(const RawMesh &raw, double cref, PreparedMesh &out, int n_threads) {
    const int threads = pick_threads(n_threads);
    const int32_t nE = raw.n_elems();
    const int32_t nN = raw.n_nodes();
    if (nE <= 0) throw std::runtime_error("mesh has no volume elements");
    if ((int64_t)raw.elem_ptr.size() != (int64_t)nE + 1) throw std::runtime_error("elem_ptr size mismatch");

    // ---- element -> local-face slots (the reference's element2faceStart, Connectivity.cpp:73-80)
    std::vector<int32_t> slot_ptr(nE + 1, 0);
    std::vector<const ElemType *> types(nE);
    for (int32_t e = 0; e < nE; e++) {
        const ElemType *t = elem_type(raw.elem_vtk[e]);
        if (!t) throw std::runtime_error("unsupported volume element VTK type " + std::to_string(raw.elem_vtk[e]) +
                                         " (supported: 10 tetra, 12 hexa, 13 wedge, 14 pyramid)");
        if (raw.elem_ptr[e + 1] - raw.elem_ptr[e] != t->n_nodes)
            throw std::runtime_error("element " + std::to_string(e) + " has the wrong node count for its type");
        types[e] = t;
        slot_ptr[e + 1] = slot_ptr[e] + t->n_faces;
    }
    for (int32_t n : raw.elem_nodes)
        if (n < 0 || n >= nN) throw std::runtime_error("element node index out of range");
    const int64_t nS = slot_ptr[nE];
    if (nS >= (int64_t)1 << 31) throw std::runtime_error("mesh too large for 32-bit face indices");

    auto slot_nodes = [&](int32_t e, int lf, int32_t *dst) {
        const ElemType *t = types[e];
        const int32_t *en = raw.elem_nodes.data() + raw.elem_ptr[e];
        for (int i = 0; i < t->face_nodes[lf]; i++) dst[i] = en[t->face_local[lf][i]];
        return t->face_nodes[lf];
    };
    std::vector<int32_t> slot_elem(nS);
    for (int32_t e = 0; e < nE; e++)
        for (int32_t s = slot_ptr[e]; s < slot_ptr[e + 1]; s++) slot_elem[s] = e;
    auto slot_key = [&](int64_t s) {
        int32_t e = slot_elem[s];
        int32_t nodes[4];
        int n = slot_nodes(e, (int)(s - slot_ptr[e]), nodes);
        return make_key(nodes, n);
    };

    // ---- match local faces: bucket slots by their smallest node, then sort inside buckets
    std::vector<int32_t> bucket_ptr(nN + 1, 0);
    std::vector<int32_t> smin(nS);
    parallel_for(nS, threads, [&](int64_t b, int64_t e) {
        for (int64_t s = b; s < e; s++) smin[s] = key_min(slot_key(s));
    });
    for (int64_t s = 0; s < nS; s++) bucket_ptr[smin[s] + 1]++;
    for (int32_t n = 0; n < nN; n++) bucket_ptr[n + 1] += bucket_ptr[n];
    std::vector<int32_t> bucket(nS);
    {
        std::vector<int32_t> cur(bucket_ptr.begin(), bucket_ptr.end() - 1);
        for (int64_t s = 0; s < nS; s++) bucket[cur[smin[s]]++] = (int32_t)s;  // slots ascending per bucket
    }
    std::vector<int32_t>().swap(smin);
    std::vector<int32_t> partner(nS, -1);
    std::vector<char> bad(threads, 0);
    parallel_for(nN, threads, [&](int64_t b, int64_t e) {
        std::vector<std::pair<Key, int32_t>> local;
        for (int64_t n = b; n < e; n++) {
            int32_t lo = bucket_ptr[n], hi = bucket_ptr[n + 1];
            if (hi - lo < 2) continue;
            local.clear();
            for (int32_t i = lo; i < hi; i++) local.emplace_back(slot_key(bucket[i]), bucket[i]);
            std::sort(local.begin(), local.end());
            for (size_t i = 0; i + 1 < local.size(); i++) {
                if (local[i].first != local[i + 1].first) continue;
                if (i + 2 < local.size() && local[i + 2].first == local[i].first) {
                    bad[0] = 1;  // a face shared by three or more elements
                    continue;
                }
                partner[local[i].second] = local[i + 1].second;
                partner[local[i + 1].second] = local[i].second;
                i++;
            }
        }
    });
    if (bad[0]) throw std::runtime_error("non-manifold mesh: a face is shared by more than two elements");
    std::vector<int32_t>().swap(bucket);
    std::vector<int32_t>().swap(bucket_ptr);

    // ---- face numbering (Connectivity.cpp:110-260): interior faces by first encounter over
    // (element, local face), then boundary faces in slot order with their ghost cells.
    std::vector<int32_t> slot_face(nS, -1);
    int32_t n_int = 0;
    for (int64_t s = 0; s < nS; s++) {
        int32_t p = partner[s];
        if (p > s) {
            slot_face[s] = n_int;
            slot_face[p] = n_int;
            n_int++;
        }
    }
    int32_t n_face = n_int;
    for (int64_t s = 0; s < nS; s++)
        if (partner[s] < 0) slot_face[s] = n_face++;
    const int32_t n_bnd = n_face - n_int;

    out = PreparedMesh();
    out.n_cells = nE;
    out.n_faces = n_face;
    out.n_faces_int = n_int;
    out.n_nodes = nN;
    out.cell2face_ptr = slot_ptr;
    out.cell2face = slot_face;
    out.cell2cell.assign(nS, -1);
    out.face2cell.assign(2 * (size_t)n_face, -1);
    out.face2node_ptr.assign((size_t)n_face + 1, 0);
    std::vector<int32_t> face_slot(n_face, -1);  // the slot whose node list the face stores
    for (int64_t s = 0; s < nS; s++) {
        int32_t f = slot_face[s];
        int32_t e = slot_elem[s];
        if (partner[s] >= 0) {
            int32_t pe = slot_elem[partner[s]];
            out.cell2cell[s] = pe;
            if (partner[s] > s) {
                out.face2cell[2 * f] = e;
                out.face2cell[2 * f + 1] = pe;
                face_slot[f] = (int32_t)s;
            }
        } else {
            int32_t ghost = nE + (f - n_int);
            out.cell2cell[s] = ghost;
            out.face2cell[2 * f] = e;
            out.face2cell[2 * f + 1] = ghost;
            face_slot[f] = (int32_t)s;
        }
    }
    for (int32_t f = 0; f < n_face; f++) {
        int32_t s = face_slot[f];
        int32_t e = slot_elem[s];
        out.face2node_ptr[f + 1] = out.face2node_ptr[f] + types[e]->face_nodes[s - slot_ptr[e]];
    }
    out.face2node.resize(out.face2node_ptr[n_face]);
    parallel_for(n_face, threads, [&](int64_t b, int64_t e) {
        for (int64_t f = b; f < e; f++) {
            int32_t s = face_slot[f];
            int32_t el = slot_elem[s];
            slot_nodes(el, s - slot_ptr[el], out.face2node.data() + out.face2node_ptr[f]);
        }
    });
    std::vector<int32_t>().swap(partner);

    // ---- metrics (Metrics.cpp:9-309) on coordinates divided by CREF (:12-19)
    std::vector<V3> P(nN);
    for (int32_t n = 0; n < nN; n++) P[n] = {raw.xyz[3 * n] / cref, raw.xyz[3 * n + 1] / cref, raw.xyz[3 * n + 2] / cref};
    out.face_normal.resize(3 * (size_t)n_face);
    out.face_unit_normal.resize(3 * (size_t)n_face);
    out.face_center.resize(3 * (size_t)n_face);
    out.face_area.resize(n_face);
    std::vector<char> badf(n_face, 0);
    parallel_for(n_face, threads, [&](int64_t b, int64_t e) {
        for (int64_t f = b; f < e; f++) {
            const int32_t *fn = out.face2node.data() + out.face2node_ptr[f];
            int nn = out.face2node_ptr[f + 1] - out.face2node_ptr[f];
            V3 c, nrm, unit;
            double area;
            if (nn == 3) {  // Metrics.cpp:96-113
                c = divs(add(add(P[fn[0]], P[fn[1]]), P[fn[2]]), 3.0);
                V3 ab = sub(P[fn[1]], P[fn[0]]), ac = sub(P[fn[2]], P[fn[0]]);
                area = tri_area(ab, ac);
                nrm = mul(cross(ab, ac), 0.5);
                unit = divs(nrm, length(nrm));
            } else {  // quad, Metrics.cpp:116-140: normal from the diagonals, "unit" = normal / area
                V3 ab = sub(P[fn[1]], P[fn[0]]), ac = sub(P[fn[2]], P[fn[0]]), ad = sub(P[fn[3]], P[fn[0]]);
                double w123 = tri_area(ab, ac), w134 = tri_area(ac, ad);
                V3 c123 = divs(add(add(P[fn[0]], P[fn[1]]), P[fn[2]]), 3.0);
                V3 c134 = divs(add(add(P[fn[0]], P[fn[2]]), P[fn[3]]), 3.0);
                c = divs(add(mul(c123, w123), mul(c134, w134)), w123 + w134);
                area = w134 + w123;
                double dxa = P[fn[3]].x - P[fn[1]].x, dxb = P[fn[2]].x - P[fn[0]].x;
                double dya = P[fn[3]].y - P[fn[1]].y, dyb = P[fn[2]].y - P[fn[0]].y;
                double dza = P[fn[3]].z - P[fn[1]].z, dzb = P[fn[2]].z - P[fn[0]].z;
                nrm = mul(V3{dza * dyb - dya * dzb, dxa * dzb - dza * dxb, dya * dxb - dxa * dyb}, 0.5);
                unit = divs(nrm, area);
            }
            if (!(area > 0.0)) badf[f] = 1;
            out.face_area[f] = area;
            std::memcpy(&out.face_center[3 * f], &c, sizeof c);
            std::memcpy(&out.face_normal[3 * f], &nrm, sizeof nrm);
            std::memcpy(&out.face_unit_normal[3 * f], &unit, sizeof unit);
        }
    });
    for (int32_t f = 0; f < n_face; f++)
        if (badf[f]) throw std::runtime_error("degenerate face " + std::to_string(f) + " (zero area)");

    out.cell_volume.resize(nE);
    out.cell_centroid.resize(3 * (size_t)nE);
    parallel_for(nE, threads, [&](int64_t b, int64_t e) {
        for (int64_t el = b; el < e; el++) {
            const int32_t *en = raw.elem_nodes.data() + raw.elem_ptr[el];
            const V3 *p[8];
            for (int i = 0; i < types[el]->n_nodes; i++) p[i] = &P[en[i]];
            double vol;
            V3 c;
            switch (types[el]->vtk) {
                case 12: {  // Metrics.cpp:184-210: area of face 0123 times |P0 - P4|
                    V3 ab = sub(*p[1], *p[0]), ac = sub(*p[2], *p[0]), ad = sub(*p[3], *p[0]);
                    double a = tri_area(ab, ac) + tri_area(ac, ad);
                    vol = a * length(sub(*p[0], *p[4]));
                    double sx = 0.0, sy = 0.0, sz = 0.0;
                    for (int i = 0; i < 8; i++) {
                        sx += p[i]->x;
                        sy += p[i]->y;
                        sz += p[i]->z;
                    }
                    c = {sx / 8.0, sy / 8.0, sz / 8.0};
                    break;
                }
                case 13: {  // Metrics.cpp:214-227: three tetrahedra
                    double v1 = tet_volume(*p[0], *p[1], *p[2], *p[3]);
                    double v2 = tet_volume(*p[1], *p[4], *p[2], *p[3]);
                    double v3 = tet_volume(*p[3], *p[5], *p[4], *p[2]);
                    vol = v1 + v2 + v3;
                    V3 c1 = tet_centroid(*p[0], *p[1], *p[2], *p[3]);
                    V3 c2 = tet_centroid(*p[1], *p[2], *p[4], *p[3]);
                    V3 c3 = tet_centroid(*p[3], *p[4], *p[5], *p[2]);
                    c = divs(add(add(mul(c1, v1), mul(c2, v2)), mul(c3, v3)), vol);
                    break;
                }
                case 14: {  // Metrics.cpp:230-240: two tetrahedra
                    double v1 = tet_volume(*p[0], *p[2], *p[3], *p[4]);
                    double v2 = tet_volume(*p[0], *p[1], *p[2], *p[4]);
                    vol = v1 + v2;
                    V3 c1 = tet_centroid(*p[0], *p[2], *p[3], *p[4]);
                    V3 c2 = tet_centroid(*p[0], *p[1], *p[2], *p[4]);
                    c = divs(add(mul(c1, v1), mul(c2, v2)), vol);
                    break;
                }
                default: {  // tetrahedron, Metrics.cpp:244-257
                    V3 s{0.0, 0.0, 0.0};
                    for (int i = 0; i < 4; i++) s = add(s, *p[i]);
                    c = divs(s, 4.0);
                    vol = tet_volume(*p[0], *p[1], *p[2], *p[3]);
                    break;
                }
            }
            out.cell_volume[el] = vol;
            std::memcpy(&out.cell_centroid[3 * el], &c, sizeof c);
        }
    });
    for (int32_t e = 0; e < nE; e++)
        if (!(out.cell_volume[e] > 0.0)) throw std::runtime_error("degenerate cell " + std::to_string(e) + " (volume not > 0)");

    // ---- orient normals from the left cell outward (Metrics::reorientFaceVectors, Metrics.cpp:270-309)
    parallel_for(n_face, threads, [&](int64_t b, int64_t e) {
        for (int64_t f = b; f < e; f++) {
            int32_t e0 = out.face2cell[2 * f], e1 = out.face2cell[2 * f + 1];
            V3 fc{out.face_center[3 * f], out.face_center[3 * f + 1], out.face_center[3 * f + 2]};
            V3 nrm{out.face_normal[3 * f], out.face_normal[3 * f + 1], out.face_normal[3 * f + 2]};
            V3 c0{out.cell_centroid[3 * e0], out.cell_centroid[3 * e0 + 1], out.cell_centroid[3 * e0 + 2]};
            double cos0 = dot(sub(c0, fc), nrm);
            bool flip;
            if (e1 < nE) {
                V3 c1{out.cell_centroid[3 * e1], out.cell_centroid[3 * e1 + 1], out.cell_centroid[3 * e1 + 2]};
                double cos1 = dot(sub(c1, fc), nrm);
                flip = cos0 > 0 && cos1 < 0;
            } else {
                flip = cos0 > 0;
            }
            if (flip)
                for (int k = 0; k < 3; k++) {
                    out.face_normal[3 * f + k] *= -1;
                    out.face_unit_normal[3 * f + k] *= -1;
                }
        }
    });

    // ---- ghost classification (Mesh::update{Wall,Farfield,Symmetry}GhostCell, Mesh.hpp:594-707):
    // every marker face is matched to the boundary face with the same node set; wall markers
    // ("wall"/"airfoil") first, then "farfield", then "sym", each in marker order.
    std::unordered_map<Key, int32_t, KeyHash> bface;
    bface.reserve((size_t)n_bnd * 2);
    for (int32_t f = n_int; f < n_face; f++) {
        const int32_t *fn = out.face2node.data() + out.face2node_ptr[f];
        bface.emplace(make_key(fn, out.face2node_ptr[f + 1] - out.face2node_ptr[f]), f);
    }
    std::vector<char> claimed(n_bnd, 0);
    auto classify = [&](auto is_kind, std::vector<int32_t> &g, std::vector<int32_t> &in, std::vector<int32_t> &fc) {
        for (const RawMarker &m : raw.markers) {
            std::string tag = m.tag;
            std::transform(tag.begin(), tag.end(), tag.begin(), [](unsigned char ch) { return (char)std::tolower(ch); });
            if (!is_kind(tag)) continue;
            for (size_t i = 0; i + 1 < m.node_ptr.size(); i++) {
                int n = m.node_ptr[i + 1] - m.node_ptr[i];
                if (n != 3 && n != 4) throw std::runtime_error("marker '" + m.tag + "' has a face that is not a triangle or quad");
                auto it = bface.find(make_key(m.nodes.data() + m.node_ptr[i], n));
                if (it == bface.end()) continue;  // the reference silently skips unmatched marker faces
                int32_t f = it->second;
                if (claimed[f - n_int])
                    throw std::runtime_error("boundary face " + std::to_string(f) + " appears in more than one marker");
                claimed[f - n_int] = 1;
                g.push_back(out.face2cell[2 * f + 1]);
                in.push_back(out.face2cell[2 * f]);
                fc.push_back(f);
            }
        }
    };
    classify([](const std::string &t) { return t == "airfoil" || t == "wall"; }, out.wall_ghost, out.wall_interior,
             out.wall_face);
    classify([](const std::string &t) { return t == "farfield"; }, out.farfield_ghost, out.farfield_interior,
             out.farfield_face);
    classify([](const std::string &t) { return t == "sym"; }, out.sym_ghost, out.sym_interior, out.sym_face);
}

// ------------------------------------------------------------------------------------ SU2 reader
namespace {

struct LineReader {
    std::ifstream in;
    std::string line;
    explicit LineReader(const std::string &p) : in(p) {}
    bool next() { return (bool)std::getline(in, line); }
};

// Value after "KEY=" on a line, or nullptr when the line does not hold KEY=.
const char *value_after(const std::string &line, const char *key) {
    size_t pos = line.find(key);
    if (pos == std::string::npos) return nullptr;
    return line.c_str() + pos + std::strlen(key);
}

int surface_nodes(int vtk) {
    switch (vtk) {
        case 5: return 3;
        case 9:
        case 8: return 4;
        default: return -1;
    }
}

}  // namespace

static void read_su2_impl(const std::string &path, RawMesh &out, std::vector<PartitionInterface> *interfaces) {
    LineReader r(path);
    if (!r.in) throw std::runtime_error("cannot open mesh file " + path);
    out = RawMesh();
    auto seek_key = [&](const char *key) -> long {
        while (r.next()) {
            const char *v = value_after(r.line, key);
            if (v) return std::strtol(v, nullptr, 10);
        }
        throw std::runtime_error(std::string("keyword \"") + key + "\" not found in " + path);
    };
    if (seek_key("NDIME=") != 3) throw std::runtime_error("mesh is not 3D (NDIME != 3)");
    long ne = seek_key("NELEM=");
    out.elem_vtk.reserve(ne);
    out.elem_ptr.reserve(ne + 1);
    out.elem_ptr.push_back(0);
    for (long i = 0; i < ne; i++) {
        if (!r.next()) throw std::runtime_error("unexpected end of file in NELEM section");
        char *p = const_cast<char *>(r.line.c_str());
        int vtk = (int)std::strtol(p, &p, 10);
        const ElemType *t = elem_type(vtk);
        if (!t) throw std::runtime_error("unsupported volume element VTK type " + std::to_string(vtk));
        for (int k = 0; k < t->n_nodes; k++) out.elem_nodes.push_back((int32_t)std::strtol(p, &p, 10));
        out.elem_vtk.push_back(vtk);
        out.elem_ptr.push_back((int32_t)out.elem_nodes.size());
    }
    long np = seek_key("NPOIN=");
    out.xyz.reserve(3 * np);
    for (long i = 0; i < np; i++) {
        if (!r.next()) throw std::runtime_error("unexpected end of file in NPOIN section");
        char *p = const_cast<char *>(r.line.c_str());
        for (int k = 0; k < 3; k++) out.xyz.push_back(std::strtod(p, &p));
    }
    long nm = seek_key("NMARK=");
    for (long m = 0; m < nm; m++) {
        RawMarker mk;
        if (!r.next()) throw std::runtime_error("unexpected end of file in NMARK section");
        const char *tv = value_after(r.line, "MARKER_TAG=");
        if (!tv) throw std::runtime_error("expected MARKER_TAG= in " + path);
        char tag[256] = {0};
        if (std::sscanf(tv, "%255s", tag) != 1) throw std::runtime_error("empty MARKER_TAG in " + path);
        mk.tag = tag;
        if (!r.next()) throw std::runtime_error("unexpected end of file after MARKER_TAG");
        const char *ev = value_after(r.line, "MARKER_ELEMS=");
        if (!ev) throw std::runtime_error("expected MARKER_ELEMS= in " + path);
        long k = std::strtol(ev, nullptr, 10);
        mk.node_ptr.push_back(0);
        for (long i = 0; i < k; i++) {
            if (!r.next()) throw std::runtime_error("unexpected end of file in marker " + mk.tag);
            char *p = const_cast<char *>(r.line.c_str());
            int vtk = (int)std::strtol(p, &p, 10);
            int n = surface_nodes(vtk);
            if (n < 0) throw std::runtime_error("unsupported surface element VTK type " + std::to_string(vtk));
            for (int j = 0; j < n; j++) mk.nodes.push_back((int32_t)std::strtol(p, &p, 10));
            mk.vtk.push_back(vtk);
            mk.node_ptr.push_back((int32_t)mk.nodes.size());
        }
        out.markers.push_back(std::move(mk));
    }
    // A .par file ends with the inter-partition markers (MeshPartition::parseMpiBoundaryElement)
    while (r.next()) {
        const char *v = value_after(r.line, "NINTERNAL_MARKER=");
        if (!v) continue;
        const long n_adj = std::strtol(v, nullptr, 10);
        if (n_adj == 0) break;
        if (!interfaces)
            throw std::runtime_error("partition file " + path + " has inter-partition markers; give the whole mesh "
                                     "or every partition");
        for (long a = 0; a < n_adj; a++) {
            PartitionInterface itf;
            if (!r.next()) throw std::runtime_error("unexpected end of file in NINTERNAL_MARKER section");
            const char *pv = value_after(r.line, "INTERNAL_MARKER=");
            if (!pv) throw std::runtime_error("expected INTERNAL_MARKER= in " + path);
            itf.other = (int32_t)std::strtol(pv, nullptr, 10);
            if (!r.next()) throw std::runtime_error("unexpected end of file after INTERNAL_MARKER");
            const char *nv = value_after(r.line, "NELEM_MPI=");
            if (!nv) throw std::runtime_error("expected NELEM_MPI= in " + path);
            const long k = std::strtol(nv, nullptr, 10);
            for (long i = 0; i < k; i++) {
                if (!r.next()) throw std::runtime_error("unexpected end of file in NELEM_MPI section");
                char *p = const_cast<char *>(r.line.c_str());
                itf.this_elem.push_back((int32_t)std::strtol(p, &p, 10));
                itf.other_elem.push_back((int32_t)std::strtol(p, &p, 10));
                const int vtk = (int)std::strtol(p, &p, 10);
                const int n = surface_nodes(vtk);
                if (n < 0) throw std::runtime_error("unsupported inter-partition face VTK type " + std::to_string(vtk));
                for (int j = 0; j < n; j++) itf.nodes.push_back((int32_t)std::strtol(p, &p, 10));
                itf.vtk.push_back(vtk);
                itf.node_ptr.push_back((int32_t)itf.nodes.size());
            }
            interfaces->push_back(std::move(itf));
        }
        break;
    }
}

void read_su2(const std::string &path, RawMesh &out) { read_su2_impl(path, out, nullptr); }

void read_su2_partition(const std::string &path, RawMesh &out, std::vector<PartitionInterface> &interfaces) {
    interfaces.clear();
    read_su2_impl(path, out, &interfaces);
}

void merge_partitions(const std::vector<RawMesh> &parts, const std::vector<std::vector<PartitionInterface>> &ifc,
                      RawMesh &out, std::vector<int32_t> &cell_ptr) {
    const int P = (int)parts.size();
    if (P == 0 || (int)ifc.size() != P) throw std::runtime_error("no partitions to merge");
    std::vector<int64_t> noff(P + 1, 0);
    for (int p = 0; p < P; p++) noff[p + 1] = noff[p] + parts[p].n_nodes();
    if (noff[P] > INT32_MAX) throw std::runtime_error("too many nodes");
    // union-find over every partition's local nodes
    std::vector<int32_t> up(noff[P]);
    std::iota(up.begin(), up.end(), 0);
    auto find = [&](int32_t x) {
        while (up[x] != x) {
            up[x] = up[up[x]];
            x = up[x];
        }
        return x;
    };
    auto bad = [](const std::string &m) { throw std::runtime_error("inconsistent partitions: " + m); };
    for (int p = 0; p < P; p++) {
        for (const PartitionInterface &I : ifc[p]) {
            const int q = I.other;
            if (q < 0 || q >= P || q == p) bad("neighbour partition " + std::to_string(q) + " out of range");
            if (q < p) continue;  // each pair once, from its lower partition
            const PartitionInterface *J = nullptr;
            for (const PartitionInterface &c : ifc[q])
                if (c.other == p) J = &c;
            if (!J) bad("partition " + std::to_string(q) + " lists no faces shared with " + std::to_string(p));
            if (J->vtk.size() != I.vtk.size())
                bad("partitions " + std::to_string(p) + " and " + std::to_string(q) + " list different face counts");
            for (size_t k = 0; k < I.vtk.size(); k++) {
                if (I.this_elem[k] != J->other_elem[k] || I.other_elem[k] != J->this_elem[k] || I.vtk[k] != J->vtk[k])
                    bad("face " + std::to_string(k) + " between partitions " + std::to_string(p) + " and " +
                        std::to_string(q) + " does not match");
                if (I.this_elem[k] < 0 || I.this_elem[k] >= parts[p].n_elems() || I.other_elem[k] < 0 ||
                    I.other_elem[k] >= parts[q].n_elems())
                    bad("inter-partition element id out of range");
                for (int i = I.node_ptr[k], j = J->node_ptr[k]; i < I.node_ptr[k + 1]; i++, j++) {
                    const int32_t a = I.nodes[i], b = J->nodes[j];
                    if (a < 0 || a >= parts[p].n_nodes() || b < 0 || b >= parts[q].n_nodes())
                        bad("inter-partition node id out of range");
                    const int32_t ra = find((int32_t)(noff[p] + a)), rb = find((int32_t)(noff[q] + b));
                    if (ra != rb) up[std::max(ra, rb)] = std::min(ra, rb);
                }
            }
        }
    }
    // merged nodes in order of first appearance (partition 0's first); duplicates must agree
    out = RawMesh();
    std::vector<int32_t> id(noff[P], -1), merged(noff[P]);
    for (int p = 0; p < P; p++)
        for (int32_t i = 0; i < parts[p].n_nodes(); i++) {
            const int32_t g = (int32_t)(noff[p] + i), r = find(g);
            if (id[r] < 0) {
                id[r] = out.n_nodes();
                for (int k = 0; k < 3; k++) out.xyz.push_back(parts[p].xyz[3 * (size_t)i + k]);
            } else {
                for (int k = 0; k < 3; k++)
                    if (out.xyz[3 * (size_t)id[r] + k] != parts[p].xyz[3 * (size_t)i + k])
                        bad("a node shared by two partitions has two different coordinates");
            }
            merged[g] = id[r];
        }
    // elements partition by partition, markers merged by tag (first-appearance order)
    cell_ptr.assign(1, 0);
    out.elem_ptr.assign(1, 0);
    std::vector<std::string> tags;
    for (int p = 0; p < P; p++) {
        const RawMesh &m = parts[p];
        for (int32_t e = 0; e < m.n_elems(); e++) {
            out.elem_vtk.push_back(m.elem_vtk[e]);
            for (int32_t k = m.elem_ptr[e]; k < m.elem_ptr[e + 1]; k++) {
                const int32_t n = m.elem_nodes[k];
                if (n < 0 || n >= m.n_nodes()) bad("element node id out of range");
                out.elem_nodes.push_back(merged[noff[p] + n]);
            }
            out.elem_ptr.push_back((int32_t)out.elem_nodes.size());
        }
        cell_ptr.push_back(out.n_elems());
        for (const RawMarker &mk : m.markers) {
            size_t t = 0;
            while (t < tags.size() && tags[t] != mk.tag) t++;
            if (t == tags.size()) {
                tags.push_back(mk.tag);
                RawMarker nm;
                nm.tag = mk.tag;
                nm.node_ptr.push_back(0);
                out.markers.push_back(std::move(nm));
            }
            RawMarker &dst = out.markers[t];
            for (size_t e = 0; e < mk.vtk.size(); e++) {
                dst.vtk.push_back(mk.vtk[e]);
                for (int32_t k = mk.node_ptr[e]; k < mk.node_ptr[e + 1]; k++) {
                    const int32_t n = mk.nodes[k];
                    if (n < 0 || n >= m.n_nodes()) bad("marker node id out of range");
                    dst.nodes.push_back(merged[noff[p] + n]);
                }
                dst.node_ptr.push_back((int32_t)dst.nodes.size());
            }
        }
    }
}

}  // namespace e3d
