"""AUSM (Liou & Steffen 1993).  The reference declares the scheme but never defines it, so there is
no reference output to match: these are the method's own properties, checked on the CPU oracle's
restatement (the GPU kernels are then compared with that restatement in test_gpu_parity.py)."""
import ctypes as C

import numpy as np

import pyoracle as po
from cases import CASES, prepared
from euler3d_b200 import meshgen as mg
from euler3d_b200.solver import Mesh


def one_face_mesh(normal):
    """Two cells sharing face 0 with the given unit normal (a minimal oracle mesh)."""
    n = np.asarray(normal, float)
    return po.Mesh({"n_cells": 2, "n_faces": 1, "n_faces_int": 1, "face2cell": np.array([0, 1], np.int32),
                    "face_unit_normal": n, "face_normal": n, "face_area": np.ones(1), "face_center": np.zeros(3),
                    "cell_volume": np.ones(2), "cell2face_ptr": np.array([0, 1, 2], np.int32),
                    "cell2face": np.array([0, 0], np.int32)})


def state(m, rows):
    s = po.State(m)
    for i, (rho, u, v, w, p) in enumerate(rows):
        q2 = u * u + v * v + w * w
        E = p / (0.4 * rho) + q2 / 2
        for k, val in zip(po.STATE_KEYS, (rho, u, v, w, p, E, E + p / rho, 0.0)):
            s.a[k][i] = val
    return s


def ausm(m, fl, s):
    F = np.zeros(5)
    po.lib().orc_ausm(C.byref(m.c), C.byref(fl), C.byref(s.c), 0, F.ctypes.data_as(C.POINTER(C.c_double)))
    return F


def test_consistency_with_the_physical_flux():
    rng = np.random.default_rng(0)
    fl = po.flow(0.7, scheme=1)
    for _ in range(50):
        n = rng.normal(size=3)
        n /= np.linalg.norm(n)
        m = one_face_mesh(n)
        rho, p = rng.uniform(0.5, 2.0, 2)
        u = rng.uniform(-2.5, 2.5, 3)  # sub- and supersonic
        s = state(m, [(rho, *u, p), (rho, *u, p)])
        V = u @ n
        H = s.a["H"][0]
        exact = np.array([rho * V, rho * V * u[0] + p * n[0], rho * V * u[1] + p * n[1], rho * V * u[2] + p * n[2],
                          rho * V * H])
        assert np.allclose(ausm(m, fl, s), exact, rtol=1e-13, atol=1e-13)


def test_supersonic_upwinding():
    """Fully supersonic to the right: the flux is the left state's physical flux."""
    n = np.array([1.0, 0.0, 0.0])
    m = one_face_mesh(n)
    fl = po.flow(2.0, scheme=1)
    s = state(m, [(1.0, 3.0, 0.2, 0.0, 1.0), (0.8, 2.5, -0.1, 0.3, 1.3)])
    rho, u, p, H = 1.0, 3.0, 1.0, s.a["H"][0]
    F = ausm(m, fl, s)
    assert np.allclose(F, [rho * u, rho * u * u + p, rho * u * 0.2, 0.0, rho * u * H], rtol=1e-14)


def test_freestream_preserved():
    raw = mg.bump_channel(6, 4, 3, jitter=0.05, seed=9, bump=1e-9)
    for mk in raw.markers:
        mk.tag = "farfield"
    m = po.Mesh(Mesh.from_raw(raw).arrays())
    fl = po.flow(0.5, 3.0, 1.4, 1.0, scheme=1)
    s = po.freestream(m, fl)
    po.update_bc(m, fl, s)
    assert np.max(np.abs(po.compute_residual(m, fl, s))) < 1e-12


def test_converged_forces_close_to_roe():
    """Both first-order schemes converge to the same flow up to discretisation error: on the
    64x32x2 channel the bump's lift agrees within 12 % and the density field within 5 %."""
    name = "c1"
    arrays = prepared(name)
    m = po.Mesh(arrays)
    out = {}
    for scheme in (0, 1):
        fl = po.flow(0.5, 0.0, 1.4, 1.5, scheme=scheme)
        s = po.freestream(m, fl)
        _, h0 = po.run(m, fl, s, 1)
        s = po.freestream(m, fl)
        st, _ = po.run(m, fl, s, 20000, min_residual=h0[0] * 1e-4)
        assert st.converged == 1
        out[scheme] = (po.aero(m, fl, s)[0], s.a["rho"][: m.n_cells].copy())
    (f0, r0), (f1, r1) = out[0], out[1]
    assert abs(f1[1] - f0[1]) / abs(f0[1]) < 0.12
    assert np.sign(f1[0]) == np.sign(f0[0])
    assert np.max(np.abs(r1 - r0) / r0) < 0.05
