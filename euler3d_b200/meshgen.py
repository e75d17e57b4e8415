"""Seeded synthetic meshes for the Euler3D explicit solver, plus SU2 / .par / .e3d writers.

The reference ships no meshes for its solver path (its two example meshes are
absent), so the workloads are generated here with the shapes, sizes and
jitter the benchmark configurations name:

* ``bump_channel``   3D channel with a 10%-thick circular-arc bump on the floor,
                     structured hexahedra (64x32x2 = 4,096 cells by default).
* ``biconvex_ogrid`` 10%-thick biconvex airfoil in an O-grid, each hexahedron
                     split into 2 prisms (256x128x4x2 = 262,144 cells by default).
* ``bump_box_tets``  box with a Gaussian bump on the floor, each hexahedron split
                     into 6 tetrahedra (128^3 x 6 = 12,582,912 cells by default).

A mesh is a :class:`RawMesh`: node coordinates, volume elements (VTK type +
node lists, the layout the reference's SU2 parser produces,
src/parser/SU2MeshParser.cpp:61-119) and boundary markers (tag + surface
elements, src/parser/SU2MeshParser.cpp:166-240).  Element order is the
generator's structured order; the solver renumbers cells internally.

Writers emit the SU2 text the reference parser reads (keyword layout from
src/parser/SU2MeshParser.cpp:39-196), the single-partition ``.par`` variant
with ``NINTERNAL_MARKER= 0`` (src/parser/MeshPartition.cpp:39-112), and the
``.e3d`` configuration (keys from src/parser/SimConfig.cpp:49-236).
Coordinates are written with 17 significant digits, so text and in-memory
meshes hold identical doubles.
"""
from __future__ import annotations

import dataclasses
import os
from typing import List, Tuple

import numpy as np

VTK_TETRA, VTK_HEXA, VTK_WEDGE, VTK_PYRAMID = 10, 12, 13, 14
VTK_TRIANGLE, VTK_QUAD = 5, 9
NODES_PER_VTK = {VTK_TETRA: 4, VTK_HEXA: 8, VTK_WEDGE: 6, VTK_PYRAMID: 5, VTK_TRIANGLE: 3, VTK_QUAD: 4}


@dataclasses.dataclass
class Marker:
    tag: str
    vtk: np.ndarray          # (k,) int32 surface VTK types
    nodes: np.ndarray        # (k, 4) int32, unused trailing entries = -1 for triangles


@dataclasses.dataclass
class RawMesh:
    xyz: np.ndarray          # (n_nodes, 3) float64
    elem_vtk: np.ndarray     # (n_elems,) int32
    elem_nodes: np.ndarray   # (n_elems, 8) int32, unused trailing entries = -1
    markers: List[Marker]
    name: str = "mesh"

    @property
    def n_cells(self) -> int:
        return int(self.elem_vtk.shape[0])

    def csr(self) -> Tuple[np.ndarray, np.ndarray]:
        """Element node lists as CSR (ptr, nodes) int32 arrays."""
        counts = np.array([NODES_PER_VTK[int(v)] for v in np.unique(self.elem_vtk)])
        lut = np.zeros(16, np.int64)
        lut[np.unique(self.elem_vtk)] = counts
        per = lut[self.elem_vtk]
        ptr = np.zeros(self.n_cells + 1, np.int64)
        np.cumsum(per, out=ptr[1:])
        mask = np.arange(8)[None, :] < per[:, None]
        return ptr.astype(np.int32), self.elem_nodes[mask].astype(np.int32)


def _pack(conn: np.ndarray, width: int) -> np.ndarray:
    out = np.full((conn.shape[0], width), -1, np.int32)
    out[:, : conn.shape[1]] = conn
    return out


def _marker(tag: str, conn: np.ndarray) -> Marker:
    k = conn.shape[1]
    vtk = VTK_TRIANGLE if k == 3 else VTK_QUAD
    return Marker(tag, np.full(conn.shape[0], vtk, np.int32), _pack(conn.astype(np.int32), 4))


# --------------------------------------------------------------------------------------------
# C1: bump channel (hexahedra)
# --------------------------------------------------------------------------------------------
def _arc_bump(x: np.ndarray, x0: float, x1: float, height: float) -> np.ndarray:
    """Circular arc through (x0,0) and (x1,0) with maximum ``height`` at mid-chord; 0 outside."""
    half = 0.5 * (x1 - x0)
    radius = (half * half + height * height) / (2.0 * height)
    xm = 0.5 * (x0 + x1)
    inside = (x > x0) & (x < x1)
    y = np.zeros_like(x)
    y[inside] = np.sqrt(radius * radius - (x[inside] - xm) ** 2) - (radius - height)
    return y


def bump_channel(nx: int = 64, ny: int = 32, nz: int = 2, jitter: float = 0.05, seed: int = 0,
                 length: float = 3.0, height: float = 1.0, depth: float = 0.1,
                 bump: float = 0.1) -> RawMesh:
    """Channel [0,length]x[0,height]x[0,depth] with a circular-arc bump of thickness ``bump``
    between x=1 and x=2 on the floor.  Interior nodes are jittered by uniform +-``jitter`` of
    the local spacing in each direction.  Tags: inlet/outlet ``farfield``, floor ``wall``,
    ceiling and z-faces ``sym``."""
    rng = np.random.default_rng(seed)
    i = np.arange(nx + 1)
    j = np.arange(ny + 1)
    k = np.arange(nz + 1)
    K, J, I = np.meshgrid(k, j, i, indexing="ij")          # node id = i + (nx+1)*(j + (ny+1)*k)
    dx = length / nx
    x = I * dx
    yb = _arc_bump(x, 1.0, 2.0, bump)
    dy = (height - yb) / ny
    y = yb + J * dy
    dz = depth / nz
    z = K * dz
    interior = (I > 0) & (I < nx) & (J > 0) & (J < ny) & (K > 0) & (K < nz)
    u = rng.uniform(-1.0, 1.0, size=(3,) + x.shape)
    x = x + np.where(interior, u[0] * jitter * dx, 0.0)
    y = y + np.where(interior, u[1] * jitter * dy, 0.0)
    z = z + np.where(interior, u[2] * jitter * dz, 0.0)
    xyz = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1).astype(np.float64)

    def nid(ii, jj, kk):
        return ii + (nx + 1) * (jj + (ny + 1) * kk)

    ck, cj, ci = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    ci, cj, ck = ci.ravel(), cj.ravel(), ck.ravel()
    hexes = np.stack([nid(ci, cj, ck), nid(ci + 1, cj, ck), nid(ci + 1, cj + 1, ck), nid(ci, cj + 1, ck),
                      nid(ci, cj, ck + 1), nid(ci + 1, cj, ck + 1), nid(ci + 1, cj + 1, ck + 1),
                      nid(ci, cj + 1, ck + 1)], axis=1)

    def quads_x(ii):
        kk, jj = np.meshgrid(np.arange(nz), np.arange(ny), indexing="ij")
        kk, jj = kk.ravel(), jj.ravel()
        return np.stack([nid(ii, jj, kk), nid(ii, jj + 1, kk), nid(ii, jj + 1, kk + 1), nid(ii, jj, kk + 1)], 1)

    def quads_y(jj):
        kk, ii = np.meshgrid(np.arange(nz), np.arange(nx), indexing="ij")
        kk, ii = kk.ravel(), ii.ravel()
        return np.stack([nid(ii, jj, kk), nid(ii + 1, jj, kk), nid(ii + 1, jj, kk + 1), nid(ii, jj, kk + 1)], 1)

    def quads_z(kk):
        jj, ii = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
        jj, ii = jj.ravel(), ii.ravel()
        return np.stack([nid(ii, jj, kk), nid(ii + 1, jj, kk), nid(ii + 1, jj + 1, kk), nid(ii, jj + 1, kk)], 1)

    markers = [
        _marker("farfield", np.concatenate([quads_x(0), quads_x(nx)])),
        _marker("wall", quads_y(0)),
        _marker("sym", np.concatenate([quads_y(ny), quads_z(0), quads_z(nz)])),
    ]
    return RawMesh(xyz, np.full(hexes.shape[0], VTK_HEXA, np.int32), _pack(hexes.astype(np.int32), 8),
                   markers, name=f"bump_channel_{nx}x{ny}x{nz}")


# --------------------------------------------------------------------------------------------
# C2: biconvex O-grid (prisms)
# --------------------------------------------------------------------------------------------
def biconvex_ogrid(ni: int = 256, nj: int = 128, nk: int = 4, jitter: float = 0.02, seed: int = 1,
                   stretch: float = 1.1, r_far: float = 30.0, thickness: float = 0.1,
                   span: float = 0.4) -> RawMesh:
    """O-grid of ``ni`` (around the wall) x ``nj`` (radial, geometric ratio ``stretch``, outer
    circle of radius ``r_far`` chords about mid-chord) x ``nk`` span layers around a biconvex
    airfoil of chord 1 and thickness ``thickness``; each hexahedron is split into 2 prisms.
    Interior nodes are jittered by +-``jitter`` of the local spacing.  Tags: airfoil
    ``airfoil``, outer boundary ``farfield``, span planes ``sym``."""
    rng = np.random.default_rng(seed)
    theta = 2.0 * np.pi * np.arange(ni) / ni
    xs = 0.5 + 0.5 * np.cos(theta)
    ts = _arc_bump(xs, 0.0, 1.0, 0.5 * thickness)
    ys = np.where(np.sin(theta) >= 0.0, ts, -ts)
    xf = 0.5 + r_far * np.cos(theta)
    yf = r_far * np.sin(theta)
    g = (stretch ** np.arange(nj + 1) - 1.0) / (stretch ** nj - 1.0)
    X = xs[None, :] + (xf - xs)[None, :] * g[:, None]       # (nj+1, ni)
    Y = ys[None, :] + (yf - ys)[None, :] * g[:, None]
    dz = span / nk
    # local in-plane spacing: shortest edge to a neighbour in i or j
    hi = np.hypot(np.roll(X, -1, 1) - X, np.roll(Y, -1, 1) - Y)
    hi = np.minimum(hi, np.roll(hi, 1, 1))
    hj = np.full_like(X, np.inf)
    dj = np.hypot(X[1:] - X[:-1], Y[1:] - Y[:-1])
    hj[:-1] = np.minimum(hj[:-1], dj)
    hj[1:] = np.minimum(hj[1:], dj)
    h = np.minimum(hi, hj)
    nodes = []
    for k in range(nk + 1):
        xk, yk = X.copy(), Y.copy()
        zk = np.full_like(X, k * dz)
        u = rng.uniform(-1.0, 1.0, size=(3,) + X.shape)
        if 0 < k < nk:
            inner = np.zeros(X.shape, bool)
            inner[1:nj, :] = True
            xk = xk + np.where(inner, u[0] * jitter * h, 0.0)
            yk = yk + np.where(inner, u[1] * jitter * h, 0.0)
            zk = zk + np.where(inner, u[2] * jitter * dz, 0.0)
        nodes.append(np.stack([xk.ravel(), yk.ravel(), zk.ravel()], 1))
    xyz = np.concatenate(nodes).astype(np.float64)

    def nid(ii, jj, kk):
        return (ii % ni) + ni * (jj + (nj + 1) * kk)

    ck, cj, ci = np.meshgrid(np.arange(nk), np.arange(nj), np.arange(ni), indexing="ij")
    ci, cj, ck = ci.ravel(), cj.ravel(), ck.ravel()
    p00, p10, p11, p01 = (ci, cj), (ci + 1, cj), (ci + 1, cj + 1), (ci, cj + 1)

    def prism(a, b, c):
        return np.stack([nid(*a, ck), nid(*b, ck), nid(*c, ck), nid(*a, ck + 1), nid(*b, ck + 1),
                         nid(*c, ck + 1)], 1)

    pa = prism(p00, p10, p11)
    pb = prism(p00, p11, p01)
    wedges = np.stack([pa, pb], 1).reshape(-1, 6)            # 2 prisms per hexahedron, adjacent ids

    kk, ii = np.meshgrid(np.arange(nk), np.arange(ni), indexing="ij")
    kk, ii = kk.ravel(), ii.ravel()
    wall = np.stack([nid(ii, 0, kk), nid(ii + 1, 0, kk), nid(ii + 1, 0, kk + 1), nid(ii, 0, kk + 1)], 1)
    far = np.stack([nid(ii, nj, kk), nid(ii + 1, nj, kk), nid(ii + 1, nj, kk + 1), nid(ii, nj, kk + 1)], 1)
    jj, ii2 = np.meshgrid(np.arange(nj), np.arange(ni), indexing="ij")
    jj, ii2 = jj.ravel(), ii2.ravel()

    def span_tris(kplane):
        ta = np.stack([nid(ii2, jj, kplane), nid(ii2 + 1, jj, kplane), nid(ii2 + 1, jj + 1, kplane)], 1)
        tb = np.stack([nid(ii2, jj, kplane), nid(ii2 + 1, jj + 1, kplane), nid(ii2, jj + 1, kplane)], 1)
        return np.stack([ta, tb], 1).reshape(-1, 3)

    markers = [
        _marker("airfoil", wall),
        _marker("farfield", far),
        _marker("sym", np.concatenate([span_tris(0), span_tris(nk)])),
    ]
    return RawMesh(xyz, np.full(wedges.shape[0], VTK_WEDGE, np.int32), _pack(wedges.astype(np.int32), 8),
                   markers, name=f"biconvex_ogrid_{ni}x{nj}x{nk}")


# --------------------------------------------------------------------------------------------
# C3: Gaussian-bump box (tetrahedra)
# --------------------------------------------------------------------------------------------
# Kuhn (Freudenthal) split of a hexahedron into 6 tetrahedra along the (0,0,0)-(1,1,1)
# diagonal: one tetrahedron per ordering of the three axes.  It is conforming between
# neighbouring hexahedra because every quad face is cut along its min-to-max diagonal.
_KUHN = [((0, 0, 0), (1, 0, 0), (1, 1, 0), (1, 1, 1)),
         ((0, 0, 0), (1, 0, 0), (1, 0, 1), (1, 1, 1)),
         ((0, 0, 0), (0, 1, 0), (1, 1, 0), (1, 1, 1)),
         ((0, 0, 0), (0, 1, 0), (0, 1, 1), (1, 1, 1)),
         ((0, 0, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1)),
         ((0, 0, 0), (0, 0, 1), (0, 1, 1), (1, 1, 1))]


def _bump_box_nodes(nx: int, ny: int, nz: int, length: float, height: float, sigma: float, jitter: float,
                    seed: int) -> np.ndarray:
    """Nodes of the bump box: an (nx+1) x (ny+1) x (nz+1) grid on [0,length]^3 whose floor (y=0)
    carries a Gaussian bump of ``height`` and width ``sigma``, interior nodes jittered by
    +-``jitter`` of the local spacing.  Node id = i + (nx+1) (j + (ny+1) k)."""
    rng = np.random.default_rng(seed)
    I = np.arange(nx + 1, dtype=np.float64)
    J = np.arange(ny + 1, dtype=np.float64)
    Kz = np.arange(nz + 1, dtype=np.float64)
    dx, dz = length / nx, length / nz
    # node id = i + (nx+1)*(j + (ny+1)*k); built plane by plane to bound memory
    xyz = np.empty(((nx + 1) * (ny + 1) * (nz + 1), 3), np.float64)
    plane = (nx + 1) * (ny + 1)
    xg = I * dx
    for kk in range(nz + 1):
        zk = kk * dz
        yb = height * np.exp(-((xg - 0.5 * length) ** 2 + (zk - 0.5 * length) ** 2) / (2.0 * sigma * sigma))
        dy = (length - yb) / ny                               # (nx+1,)
        x = np.broadcast_to(xg[None, :], (ny + 1, nx + 1)).copy()
        y = yb[None, :] + J[:, None] * dy[None, :]
        z = np.full_like(x, zk)
        u = rng.uniform(-1.0, 1.0, size=(3, ny + 1, nx + 1))
        if 0 < kk < nz:
            inner = np.zeros((ny + 1, nx + 1), bool)
            inner[1:ny, 1:nx] = True
            x += np.where(inner, u[0] * jitter * dx, 0.0)
            y += np.where(inner, u[1] * jitter * dy[None, :], 0.0)
            z += np.where(inner, u[2] * jitter * dz, 0.0)
        xyz[kk * plane:(kk + 1) * plane, 0] = x.ravel()
        xyz[kk * plane:(kk + 1) * plane, 1] = y.ravel()
        xyz[kk * plane:(kk + 1) * plane, 2] = z.ravel()
    return xyz


def bump_box_tets(n: int = 128, length: float = 4.0, height: float = 0.1, sigma: float = 0.3,
                  jitter: float = 0.03, seed: int = 2, nx: int = 0, ny: int = 0, nz: int = 0) -> RawMesh:
    """``nx x ny x nz`` (default ``n``^3) hexahedra on [0,length]^3 with a Gaussian bump of
    ``height`` and width ``sigma`` centred on the floor (y=0), each split into 6 tetrahedra.
    Interior nodes are jittered by +-``jitter`` of the local spacing.  Tags: floor ``wall``,
    inlet/outlet (x) and top (y) ``farfield``, z-faces ``sym``."""
    nx, ny, nz = nx or n, ny or n, nz or n
    xyz = _bump_box_nodes(nx, ny, nz, length, height, sigma, jitter, seed)

    def nid(ii, jj, kk):
        return ii + (nx + 1) * (jj + (ny + 1) * kk)

    ck, cj, ci = np.meshgrid(np.arange(nz, dtype=np.int64), np.arange(ny, dtype=np.int64),
                             np.arange(nx, dtype=np.int64), indexing="ij")
    ci, cj, ck = ci.ravel(), cj.ravel(), ck.ravel()
    tets = np.empty((ci.size, 6, 4), np.int32)
    for t, verts in enumerate(_KUHN):
        for v, (a, b, c) in enumerate(verts):
            tets[:, t, v] = nid(ci + a, cj + b, ck + c)
    tets = tets.reshape(-1, 4)
    del ci, cj, ck

    def split_quads(q):
        """q: (m,4) corners in cyclic order with corner 0 = min, corner 2 = max of the hex axes."""
        return np.stack([np.stack([q[:, 0], q[:, 1], q[:, 2]], 1), np.stack([q[:, 0], q[:, 2], q[:, 3]], 1)],
                        1).reshape(-1, 3)

    def face_x(ii):
        kk, jj = np.meshgrid(np.arange(nz), np.arange(ny), indexing="ij")
        kk, jj = kk.ravel(), jj.ravel()
        return split_quads(np.stack([nid(ii, jj, kk), nid(ii, jj + 1, kk), nid(ii, jj + 1, kk + 1),
                                     nid(ii, jj, kk + 1)], 1))

    def face_y(jj):
        kk, ii = np.meshgrid(np.arange(nz), np.arange(nx), indexing="ij")
        kk, ii = kk.ravel(), ii.ravel()
        return split_quads(np.stack([nid(ii, jj, kk), nid(ii + 1, jj, kk), nid(ii + 1, jj, kk + 1),
                                     nid(ii, jj, kk + 1)], 1))

    def face_z(kk):
        jj, ii = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
        jj, ii = jj.ravel(), ii.ravel()
        return split_quads(np.stack([nid(ii, jj, kk), nid(ii + 1, jj, kk), nid(ii + 1, jj + 1, kk),
                                     nid(ii, jj + 1, kk)], 1))

    markers = [
        _marker("farfield", np.concatenate([face_x(0), face_x(nx), face_y(ny)])),
        _marker("wall", face_y(0)),
        _marker("sym", np.concatenate([face_z(0), face_z(nz)])),
    ]
    return RawMesh(xyz, np.full(tets.shape[0], VTK_TETRA, np.int32), _pack(tets, 8), markers,
                   name=f"bump_box_tets_{nx}x{ny}x{nz}")


# faces of a VTK hexahedron, outward, in the reference's element definition order
# (src/mesh/Mesh.hpp element face tables)
_HEX_FACES = ((0, 3, 2, 1), (0, 1, 5, 4), (1, 2, 6, 5), (2, 3, 7, 6), (3, 0, 4, 7), (4, 5, 6, 7))


def bump_box_pyramids(n: int = 4, length: float = 4.0, height: float = 0.1, sigma: float = 0.3,
                      jitter: float = 0.03, seed: int = 2, nx: int = 0, ny: int = 0, nz: int = 0) -> RawMesh:
    """The bump box of :func:`bump_box_tets` in mixed elements: a hexahedron where i + j + k is
    even, elsewhere the hexahedron split into six pyramids, one on each of its faces, with their
    apex at a node added at its centre (the mean of its eight corners).  Every face between two
    cells of different hexahedra is a whole quadrilateral, so the mesh is conforming; the pyramids
    of one hexahedron meet on triangles.  A pyramid's base is its hexahedron face with the node
    order reversed, so that the pyramid's own base face (nodes 0 3 2 1) points outward like the
    hexahedron's.  Cells are listed hexahedron slot by slot.  Tags as in bump_box_tets."""
    nx, ny, nz = nx or n, ny or n, nz or n
    xyz = _bump_box_nodes(nx, ny, nz, length, height, sigma, jitter, seed)

    def nid(ii, jj, kk):
        return ii + (nx + 1) * (jj + (ny + 1) * kk)

    ck, cj, ci = np.meshgrid(np.arange(nz, dtype=np.int64), np.arange(ny, dtype=np.int64),
                             np.arange(nx, dtype=np.int64), indexing="ij")
    ci, cj, ck = ci.ravel(), cj.ravel(), ck.ravel()
    corners = ((0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1))
    hexes = np.stack([nid(ci + a, cj + b, ck + c) for a, b, c in corners], 1).astype(np.int32)
    split = (ci + cj + ck) % 2 == 1
    centre = xyz[hexes[split]].mean(axis=1)
    apex = xyz.shape[0] + np.arange(int(split.sum()), dtype=np.int32)
    xyz = np.concatenate([xyz, centre])
    hs = hexes[split]
    pyr = np.empty((hs.shape[0], 6, 5), np.int32)
    for f, (a, b, c, d) in enumerate(_HEX_FACES):
        pyr[:, f] = np.stack([hs[:, a], hs[:, d], hs[:, c], hs[:, b], apex], 1)
    # cells in slot order: a whole hexahedron, or the six pyramids of a split one
    slot = np.arange(ci.size)
    cells = np.concatenate([_pack(hexes[~split], 8), _pack(pyr.reshape(-1, 5), 8)])
    vtk = np.concatenate([np.full(int((~split).sum()), VTK_HEXA, np.int32),
                          np.full(pyr.shape[0] * 6, VTK_PYRAMID, np.int32)])
    order = np.argsort(np.concatenate([8 * slot[~split], ((8 * slot[split])[:, None] + np.arange(6)).ravel()]),
                       kind="stable")

    def face_x(ii):
        kk, jj = np.meshgrid(np.arange(nz), np.arange(ny), indexing="ij")
        kk, jj = kk.ravel(), jj.ravel()
        return np.stack([nid(ii, jj, kk), nid(ii, jj + 1, kk), nid(ii, jj + 1, kk + 1), nid(ii, jj, kk + 1)], 1)

    def face_y(jj):
        kk, ii = np.meshgrid(np.arange(nz), np.arange(nx), indexing="ij")
        kk, ii = kk.ravel(), ii.ravel()
        return np.stack([nid(ii, jj, kk), nid(ii + 1, jj, kk), nid(ii + 1, jj, kk + 1), nid(ii, jj, kk + 1)], 1)

    def face_z(kk):
        jj, ii = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
        jj, ii = jj.ravel(), ii.ravel()
        return np.stack([nid(ii, jj, kk), nid(ii + 1, jj, kk), nid(ii + 1, jj + 1, kk), nid(ii, jj + 1, kk)], 1)

    markers = [
        _marker("farfield", np.concatenate([face_x(0), face_x(nx), face_y(ny)])),
        _marker("wall", face_y(0)),
        _marker("sym", np.concatenate([face_z(0), face_z(nz)])),
    ]
    return RawMesh(xyz, vtk[order], cells[order], markers, name=f"bump_box_pyramids_{nx}x{ny}x{nz}")


# --------------------------------------------------------------------------------------------
# writers
# --------------------------------------------------------------------------------------------
def _write_rows(f, ids: np.ndarray, lead: np.ndarray, counts: np.ndarray) -> None:
    rows = []
    for v, row, c in zip(lead.tolist(), ids.tolist(), counts.tolist()):
        rows.append(" ".join([str(v)] + [str(x) for x in row[:c]]))
    f.write("\n".join(rows))
    f.write("\n")


def write_su2(mesh: RawMesh, path: str, partition: bool = True) -> None:
    """Write ``mesh`` as SU2 text; with ``partition`` append ``NINTERNAL_MARKER= 0`` so that the
    file is a single-partition ``.par`` file the reference solver reads directly."""
    with open(path, "w") as f:
        f.write("%\n% Problem dimension\n%\nNDIME= 3\n%\n% Inner element connectivity\n%\n")
        f.write(f"NELEM= {mesh.n_cells}\n")
        counts = np.array([NODES_PER_VTK[int(v)] for v in mesh.elem_vtk.tolist()])
        _write_rows(f, mesh.elem_nodes, mesh.elem_vtk, counts)
        f.write("%\n% Node coordinates\n%\n")
        f.write(f"NPOIN= {mesh.xyz.shape[0]}\n")
        f.write("\n".join(f"{x!r} {y!r} {z!r}" for x, y, z in mesh.xyz.tolist()))
        f.write("\n%\n% Boundary elements\n%\n")
        f.write(f"NMARK= {len(mesh.markers)}\n")
        for m in mesh.markers:
            f.write(f"MARKER_TAG= {m.tag}\n")
            f.write(f"MARKER_ELEMS= {m.vtk.shape[0]}\n")
            counts = np.array([NODES_PER_VTK[int(v)] for v in m.vtk.tolist()])
            _write_rows(f, m.nodes, m.vtk, counts)
        if partition:
            f.write("NINTERNAL_MARKER= 0\n")


def _face_keys(nodes: np.ndarray) -> np.ndarray:
    """One sortable key per face from its (k, 4) node rows (-1 padded): the sorted node ids."""
    k = np.sort(np.where(nodes < 0, np.iinfo(np.int64).max, nodes.astype(np.int64)), axis=1)
    return np.ascontiguousarray(k).view([("a", np.int64), ("b", np.int64), ("c", np.int64), ("d", np.int64)]).ravel()


def _format_rows(fmt_of_count, counts: np.ndarray, values: np.ndarray) -> str:
    """Rows of integers formatted in one pass: row i has counts[i] values and the format
    fmt_of_count[counts[i]]; ``values`` holds the rows' values back to back."""
    return "".join(fmt_of_count[c] for c in counts.tolist()) % tuple(values.tolist())


def write_partitions(mesh: RawMesh, n_parts: int, pattern: str, arrays=None) -> List[str]:
    """Split ``mesh`` into ``n_parts`` slabs along x (cells by the x of their mean node) and write
    one ``.par`` file per part in the layout of the reference's partitioner (E3D_PRE,
    src/partition/Partition.cpp:150-296, src/partition/SU2Writer.cpp): each part's elements in
    ascending global order, its nodes renumbered by first use, its boundary elements, and
    NINTERNAL_MARKER sections listing every face shared with another part -- the element on each
    side (local ids) and the face's nodes in the writing part's numbering, in the same order in both
    parts' files (the order of a loop over parts, their elements and the elements' faces).
    ``pattern`` contains ``#``, replaced by the part index (the reference's PARTITION_FILES
    convention).  Coordinates are written exactly.  ``arrays``: the mesh's prepared arrays, if the
    caller has them.  Vectorised, so that meshes of 10^7 cells are written in about a minute.
    Returns the file paths."""
    from .solver import Mesh  # the global connectivity, in the reference's numbering

    a = arrays if arrays is not None else Mesh.from_raw(mesh).arrays()
    n_cells = int(a["n_cells"])
    n_faces, n_int = int(a["n_faces"]), int(a["n_faces_int"])
    f2c = np.asarray(a["face2cell"]).reshape(-1, 2).astype(np.int64)
    c2f_ptr, c2f = np.asarray(a["cell2face_ptr"], np.int64), np.asarray(a["cell2face"], np.int64)
    f2n_ptr, f2n = np.asarray(a["face2node_ptr"], np.int64), np.asarray(a["face2node"], np.int64)
    npe = np.zeros(16, np.int64)
    for v, k in NODES_PER_VTK.items():
        npe[v] = k
    ecount = npe[mesh.elem_vtk]
    # x of each cell's mean node, as numpy's mean of the node x values computes it
    cx = np.empty(n_cells)
    xs = np.where(mesh.elem_nodes >= 0, mesh.xyz[np.maximum(mesh.elem_nodes, 0), 0], 0.0)
    for k in np.unique(ecount).tolist():
        sel = np.flatnonzero(ecount == k)
        cx[sel] = xs[sel, :k].mean(axis=1)
    part = np.empty(n_cells, np.int64)
    part[np.argsort(cx, kind="stable")] = np.arange(n_cells, dtype=np.int64) * n_parts // n_cells
    g2l = np.empty(n_cells, np.int64)
    elems = []
    for p in range(n_parts):
        e = np.flatnonzero(part == p)
        g2l[e] = np.arange(e.size)
        elems.append(e)
    # local node numbering by first use over each part's elements
    local = []   # global -> local node id of each part (-1: not in the part)
    inv = []     # local -> global
    for p in range(n_parts):
        rows = mesh.elem_nodes[elems[p]]
        seq = rows[rows >= 0]
        uniq, first = np.unique(seq, return_index=True)
        g = uniq[np.argsort(first, kind="stable")]
        m = np.full(mesh.xyz.shape[0], -1, np.int64)
        m[g] = np.arange(g.size)
        local.append(m)
        inv.append(g)
    # marker faces matched to boundary faces by node set: the part of the face's interior cell
    bnodes = np.full((n_faces - n_int, 4), -1, np.int64)
    bcount = f2n_ptr[n_int + 1:] - f2n_ptr[n_int:-1]
    for k in (3, 4):
        sel = np.flatnonzero(bcount == k)
        bnodes[sel, :k] = f2n[f2n_ptr[n_int + sel][:, None] + np.arange(k)[None, :]]
    bkey = _face_keys(bnodes)
    border = np.argsort(bkey, kind="stable")
    bsorted = bkey[border]
    mk_part = []
    for mk in mesh.markers:
        nodes = np.where(np.arange(4)[None, :] < npe[mk.vtk][:, None], mk.nodes, -1)
        key = _face_keys(nodes)
        pos = np.minimum(np.searchsorted(bsorted, key), bsorted.size - 1)
        if not np.all(bsorted[pos] == key):
            raise ValueError(f"marker {mk.tag!r} has a face that is not a boundary face")
        mk_part.append(part[f2c[n_int + border[pos], 0]])
    # inter-part faces: every (cell, face) entry whose neighbour is an interior cell of a
    # higher-numbered part, in the order of the loop over parts, elements and element faces
    cell_of = np.repeat(np.arange(n_cells), np.diff(c2f_ptr))
    fe = c2f
    other = np.where(f2c[fe, 0] == cell_of, f2c[fe, 1], f2c[fe, 0])
    inner = other < n_cells
    cross = np.flatnonzero(inner & (part[cell_of] < part[np.minimum(other, n_cells - 1)]))
    ce, co, cf = cell_of[cross], other[cross], fe[cross]
    pp, qq = part[ce], part[co]
    order = np.lexsort((cross, qq, pp))  # by (p, q), then loop order
    ce, co, cf, pp, qq = ce[order], co[order], cf[order], pp[order], qq[order]
    fcount = f2n_ptr[cf + 1] - f2n_ptr[cf]
    fnodes = np.full((cf.size, 4), -1, np.int64)
    for k in (3, 4):
        sel = np.flatnonzero(fcount == k)
        fnodes[sel, :k] = f2n[f2n_ptr[cf[sel]][:, None] + np.arange(k)[None, :]]
    fvtk = np.where(fcount == 3, 5, np.where(fcount == 4, 9, 7))

    efmt = {k: "%3d" + "%10d" * k + "%10d\n" for k in range(1, 9)}
    ifmt = {k: "%10d" * (3 + k) + "\n" for k in range(1, 5)}
    mfmt = {k: "%3d" + "%10d" * k + "\n" for k in range(1, 5)}
    paths = []
    for p in range(n_parts):
        path = pattern.replace("#", str(p))
        m = local[p]
        with open(path, "w") as f:
            f.write("%\n% Problem dimension\n%\nNDIME= 3\n%\n% Inner element connectivity\n%\n")
            e = elems[p]
            f.write(f"NELEM= {e.size}\n")
            k_e = ecount[e]
            rows = mesh.elem_nodes[e]
            vals = np.concatenate([mesh.elem_vtk[e][:, None].astype(np.int64), np.where(rows >= 0, m[np.maximum(rows, 0)], -1),
                                   np.arange(e.size)[:, None]], axis=1)
            keep = np.concatenate([np.ones((e.size, 1), bool), rows >= 0, np.ones((e.size, 1), bool)], axis=1)
            f.write(_format_rows(efmt, k_e, vals[keep]))
            f.write(f"%\n% Node coordinates\n%\nNPOIN= {inv[p].size}\n")
            xyz = mesh.xyz[inv[p]]
            vals = [x for row in zip(xyz[:, 0].tolist(), xyz[:, 1].tolist(), xyz[:, 2].tolist(), range(inv[p].size))
                    for x in row]
            f.write(("%26r%26r%26r%10d\n" * inv[p].size) % tuple(vals))
            mk_text, n_mk = [], 0
            for mk, mp in zip(mesh.markers, mk_part):
                sel = np.flatnonzero(mp == p)
                if sel.size == 0:
                    continue
                n_mk += 1
                kk = npe[mk.vtk[sel]]
                nodes = mk.nodes[sel]
                keep = np.arange(4)[None, :] < kk[:, None]
                vals = np.concatenate([mk.vtk[sel][:, None].astype(np.int64), np.where(keep, m[np.maximum(nodes, 0)], -1)],
                                      axis=1)[np.concatenate([np.ones((sel.size, 1), bool), keep], axis=1)]
                mk_text.append(f"MARKER_TAG= {mk.tag}\nMARKER_ELEMS= {sel.size}\n" + _format_rows(mfmt, kk, vals))
            f.write(f"%\n% Boundary elements\n%\nNMARK= {n_mk}\n")
            f.write("".join(mk_text))
            # this part's side of each inter-part face: rows where it is p (cells ce) or q (cells co)
            adj = sorted(set(qq[pp == p].tolist()) | set(pp[qq == p].tolist()))
            f.write(f"%\n% Internal Boundary elements\n%\nNINTERNAL_MARKER= {len(adj)}\n")
            for q in adj:
                if p < q:
                    sel = np.flatnonzero((pp == p) & (qq == q))
                    mine, theirs = ce[sel], co[sel]
                else:
                    sel = np.flatnonzero((pp == q) & (qq == p))
                    mine, theirs = co[sel], ce[sel]
                kk = fcount[sel]
                nodes = fnodes[sel]
                keep = nodes >= 0
                vals = np.concatenate([g2l[mine][:, None], g2l[theirs][:, None], fvtk[sel][:, None],
                                       np.where(keep, m[np.maximum(nodes, 0)], -1)], axis=1)
                vals = vals[np.concatenate([np.ones((sel.size, 3), bool), keep], axis=1)]
                f.write(f"INTERNAL_MARKER= {q}\nNELEM_MPI= {sel.size}\n")
                f.write(_format_rows(ifmt, kk, vals))
        paths.append(path)
    return paths


@dataclasses.dataclass
class CaseConfig:
    """Flow and solver settings written into an ``.e3d`` file (src/parser/SimConfig.cpp:49-236)."""
    mach: float = 0.5
    aoa: float = 0.0
    gamma: float = 1.4
    cfl: float = 1.5
    min_residual: float = 0.0
    min_aerocoeff_error: float = 0.0
    max_iter: int = 100
    sampling: int = 1
    scheme: int = 0
    time_integration: int = 2     # TIME_INTEGRATION=: 0 explicit Euler, 2 RK5
    residual_smoothing: int = 0   # RESIDUAL_SMOOTHING=
    orientation_cl: int = 2
    orientation_cd: int = 0
    ref_point: Tuple[float, float, float] = (0.25, 0.0, 0.0)
    sref: float = 1.0
    cref: float = 1.0


def write_e3d(cfg: CaseConfig, path: str, par_pattern: str, output_file: str, n_partitions: int = 1) -> None:
    """Write an ``.e3d`` configuration.  ``CREF``, ``SREF`` and ``RESIDUAL_SMOOTHING`` are always
    written because the reference leaves them uninitialised when absent
    (include/parser/SimConfig.hpp:149-150,179)."""
    lines = [
        "START",
        f"INITIAL_MESH= unused.su2",
        f"PARTITION_FILES= {n_partitions}",
        par_pattern,
        "PRE_LOG= prelog.txt",
        f"MESH_ORIENTATION_CL= {cfg.orientation_cl}",
        f"MESH_ORIENTATION_CD= {cfg.orientation_cd}",
        f"MESH_REF_POINT_X= {cfg.ref_point[0]!r}",
        f"MESH_REF_POINT_Y= {cfg.ref_point[1]!r}",
        f"MESH_REF_POINT_Z= {cfg.ref_point[2]!r}",
        f"SREF= {cfg.sref!r}",
        f"CREF= {cfg.cref!r}",
        f"SAMPLING= {cfg.sampling}",
        "SPEED_OPTION= 0",
        f"SPEED_VALUE= {cfg.mach!r}",
        f"AOA= {cfg.aoa!r}",
        "AIRFLOW_PRESSURE= 101325",
        "AIRFLOW_TEMPERATURE= 288.15",
        "AIRFLOW_VISCOSITY= 1.853e-5",
        "AIRFLOW_DENSITY= 1.2886",
        f"GAMMA= {cfg.gamma!r}",
        "GAS_CONSTANT= 287.058",
        "SPECIFIC_HEAT= 1004.7",
        f"SCHEME= {cfg.scheme}",
        f"TIME_INTEGRATION= {cfg.time_integration}",
        f"RESIDUAL_SMOOTHING= {cfg.residual_smoothing}",
        f"CFL= {cfg.cfl!r}",
        f"MIN_RESIDUAL= {cfg.min_residual!r}",
        f"MIN_AEROCOEFF_ERROR= {cfg.min_aerocoeff_error!r}",
        f"MAX_ITER= {cfg.max_iter}",
        "SOLVER_LOG= solverlog.txt",
        f"OUTPUT_FILE= {output_file}",
        "POST_LOG= postlog.txt",
        "END",
    ]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def write_case(mesh: RawMesh, cfg: CaseConfig, directory: str) -> str:
    """Write ``mesh.par`` and ``case.e3d`` into ``directory``; return the config path."""
    os.makedirs(os.path.join(directory, "output"), exist_ok=True)
    par = os.path.join(directory, "mesh.par")
    write_su2(mesh, par, partition=True)
    cfg_path = os.path.join(directory, "case.e3d")
    write_e3d(cfg, cfg_path, par, os.path.join(directory, "output", "out.dat"))
    return cfg_path
