"""ctypes binding of the CPU oracle (oracle/e3d_oracle.c) and of the reference checker binary.

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()`` and by the
CPU-baseline leg of ``bench.py``; never by the product package.

Meshes are passed as a dict of numpy arrays in the reference's numbering:
``n_cells n_faces n_faces_int face2cell face_unit_normal face_normal face_area face_center
cell_volume cell2face_ptr cell2face {wall,farfield,sym}_{ghost,interior,face}``.
States are dicts with ``rho u v w p E H M`` arrays of n_cells + (n_faces - n_faces_int) values.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Dict, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libe3d_oracle.so")
REF_DRIVER = os.path.join(HERE, "_ref", "e3d_ref_driver")
STATE_KEYS = ("rho", "u", "v", "w", "p", "E", "H", "M")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class OrcMesh(C.Structure):
    _fields_ = [("n_cells", C.c_int), ("n_faces", C.c_int), ("n_faces_int", C.c_int),
                ("face2cell", _ip), ("face_unit_normal", _dp), ("face_normal", _dp), ("face_area", _dp),
                ("face_center", _dp), ("cell_volume", _dp), ("cell2face_ptr", _ip), ("cell2face", _ip),
                ("n_wall", C.c_int), ("wall_ghost", _ip), ("wall_interior", _ip), ("wall_face", _ip),
                ("n_farfield", C.c_int), ("farfield_ghost", _ip), ("farfield_interior", _ip),
                ("farfield_face", _ip),
                ("n_sym", C.c_int), ("sym_ghost", _ip), ("sym_interior", _ip), ("sym_face", _ip)]


class OrcFlow(C.Structure):
    _fields_ = [("gamma", C.c_double), ("cfl", C.c_double), ("mach", C.c_double), ("aoa_deg", C.c_double),
                ("rho_inf", C.c_double), ("p_inf", C.c_double), ("u_inf", C.c_double), ("v_inf", C.c_double),
                ("w_inf", C.c_double), ("E_inf", C.c_double), ("H_inf", C.c_double), ("M_inf", C.c_double),
                ("sref", C.c_double), ("cref", C.c_double), ("ref_point", C.c_double * 3),
                ("cl_axis", C.c_int), ("cl_sign", C.c_int), ("cd_axis", C.c_int), ("cd_sign", C.c_int),
                ("cm_axis", C.c_int), ("cm_sign", C.c_int), ("scheme", C.c_int), ("integrator", C.c_int),
                ("smoothing", C.c_int)]


class OrcState(C.Structure):
    _fields_ = [(k, _dp) for k in STATE_KEYS]


class OrcRunParams(C.Structure):
    _fields_ = [("max_iter", C.c_int), ("sampling", C.c_int), ("min_residual", C.c_double),
                ("min_aerocoeff_error", C.c_double), ("rms_history", _dp)]


class OrcRunStats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("converged", C.c_int), ("n_rms", C.c_int), ("last_rms", C.c_double),
                ("cl", C.c_double), ("cd", C.c_double), ("cm", C.c_double), ("force", C.c_double * 3),
                ("moment", C.c_double * 3), ("smooth_sweeps", C.c_longlong)]


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"oracle library missing: {LIB_PATH} (run `make -C oracle port`)")
        L = C.CDLL(LIB_PATH)
        M, F, S = C.POINTER(OrcMesh), C.POINTER(OrcFlow), C.POINTER(OrcState)
        L.orc_flow_init.argtypes = [F]
        L.orc_state_freestream.argtypes = [M, F, S]
        L.orc_update_bc.argtypes = [M, F, S]
        L.orc_compute_residual.argtypes = [M, F, S, _dp]
        L.orc_time_step.argtypes = [M, F, S, _dp]
        L.orc_roe.argtypes = [M, F, S, C.c_int, _dp]
        L.orc_ausm.argtypes = [M, F, S, C.c_int, _dp]
        L.orc_runge_kutta.argtypes = [M, F, S, _dp, _dp]
        L.orc_runge_kutta.restype = C.c_longlong
        L.orc_smooth_residuals.argtypes = [M, _dp]
        L.orc_smooth_residuals.restype = C.c_longlong
        L.orc_euler_explicit.argtypes = [M, F, S, _dp, _dp, _dp]
        L.orc_rms.argtypes = [M, _dp]
        L.orc_rms.restype = C.c_double
        L.orc_aero_coefficients.argtypes = [M, F, S, _dp, _dp]
        L.orc_run.argtypes = [M, F, S, C.POINTER(OrcRunParams), C.POINTER(OrcRunStats)]
        L.orc_run.restype = C.c_int
        _lib = L
    return _lib


def _d(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def _i(a: np.ndarray):
    return a.ctypes.data_as(_ip)


class Mesh:
    """Keeps the numpy arrays alive behind an ``orc_mesh``."""

    def __init__(self, arrays: Dict[str, np.ndarray]):
        a = {}
        for k, v in arrays.items():
            if isinstance(v, np.ndarray):
                a[k] = np.ascontiguousarray(v, dtype=np.int32 if v.dtype.kind in "iu" else np.float64)
            else:
                a[k] = v
        for tag in ("wall", "farfield", "sym"):
            for part in ("ghost", "interior", "face"):
                a.setdefault(f"{tag}_{part}", np.zeros(0, np.int32))
                if a[f"{tag}_{part}"].size == 0:
                    a[f"{tag}_{part}"] = np.zeros(1, np.int32)[:0].copy()
        self.a = a
        m = OrcMesh()
        m.n_cells, m.n_faces, m.n_faces_int = int(a["n_cells"]), int(a["n_faces"]), int(a["n_faces_int"])
        m.face2cell = _i(a["face2cell"])
        for k in ("face_unit_normal", "face_normal", "face_area", "face_center", "cell_volume"):
            setattr(m, k, _d(a[k]))
        m.cell2face_ptr, m.cell2face = _i(a["cell2face_ptr"]), _i(a["cell2face"])
        for tag in ("wall", "farfield", "sym"):
            setattr(m, f"n_{tag}", int(a[f"{tag}_ghost"].size))
            for part in ("ghost", "interior", "face"):
                setattr(m, f"{tag}_{part}", _i(a[f"{tag}_{part}"]))
        self.c = m

    @property
    def n_cells(self) -> int:
        return int(self.a["n_cells"])

    @property
    def n_total(self) -> int:
        return int(self.a["n_cells"]) + int(self.a["n_faces"]) - int(self.a["n_faces_int"])


def flow(mach: float, aoa: float = 0.0, gamma: float = 1.4, cfl: float = 1.5, sref: float = 1.0,
         cref: float = 1.0, ref_point=(0.25, 0.0, 0.0), cl=(1, 1), cd=(0, 1), cm=(2, 1), scheme: int = 0,
         integrator: int = 0, smoothing: bool = False) -> OrcFlow:
    """Flow settings; ``integrator`` 0 is RK5 (TIME_INTEGRATION= 2), 1 explicit Euler (TIME_INTEGRATION= 0)."""
    f = OrcFlow()
    f.scheme = scheme
    f.integrator, f.smoothing = integrator, int(bool(smoothing))
    f.gamma, f.cfl, f.mach, f.aoa_deg = gamma, cfl, mach, aoa
    f.sref, f.cref = sref, cref
    f.ref_point[:] = list(ref_point)
    f.cl_axis, f.cl_sign = cl
    f.cd_axis, f.cd_sign = cd
    f.cm_axis, f.cm_sign = cm
    lib().orc_flow_init(C.byref(f))
    return f


class State:
    def __init__(self, mesh: Mesh, arrays: Optional[Dict[str, np.ndarray]] = None):
        n = mesh.n_total
        self.a = {k: np.zeros(n) for k in STATE_KEYS}
        if arrays is not None:
            for k in STATE_KEYS:
                self.a[k][:] = arrays[k]
        self.c = OrcState(*[_d(self.a[k]) for k in STATE_KEYS])

    def copy(self, mesh: Mesh) -> "State":
        return State(mesh, self.a)


def freestream(mesh: Mesh, fl: OrcFlow) -> State:
    s = State(mesh)
    lib().orc_state_freestream(C.byref(mesh.c), C.byref(fl), C.byref(s.c))
    return s


def update_bc(mesh: Mesh, fl: OrcFlow, s: State) -> None:
    lib().orc_update_bc(C.byref(mesh.c), C.byref(fl), C.byref(s.c))


def compute_residual(mesh: Mesh, fl: OrcFlow, s: State) -> np.ndarray:
    R = np.zeros(5 * mesh.n_cells)
    lib().orc_compute_residual(C.byref(mesh.c), C.byref(fl), C.byref(s.c), _d(R))
    return R.reshape(-1, 5)


def time_step(mesh: Mesh, fl: OrcFlow, s: State) -> np.ndarray:
    dt = np.zeros(mesh.n_cells)
    lib().orc_time_step(C.byref(mesh.c), C.byref(fl), C.byref(s.c), _d(dt))
    return dt


def runge_kutta(mesh: Mesh, fl: OrcFlow, s: State, R: np.ndarray) -> np.ndarray:
    R = np.ascontiguousarray(R, dtype=np.float64).reshape(-1).copy()
    dt = np.zeros(mesh.n_cells)
    lib().orc_runge_kutta(C.byref(mesh.c), C.byref(fl), C.byref(s.c), _d(R), _d(dt))
    return R.reshape(-1, 5)


def smooth_residuals(mesh: Mesh, R: np.ndarray):
    """EulerSolver::smoothResiduals on a copy of R; returns (smoothed R [n, 5], sweeps or -1)."""
    R = np.ascontiguousarray(R, dtype=np.float64).reshape(-1).copy()
    n = lib().orc_smooth_residuals(C.byref(mesh.c), _d(R))
    return R.reshape(-1, 5), int(n)


def rms(mesh: Mesh, R: np.ndarray) -> float:
    R = np.ascontiguousarray(R, dtype=np.float64).reshape(-1)
    return float(lib().orc_rms(C.byref(mesh.c), _d(R)))


def aero(mesh: Mesh, fl: OrcFlow, s: State):
    f, m = np.zeros(3), np.zeros(3)
    lib().orc_aero_coefficients(C.byref(mesh.c), C.byref(fl), C.byref(s.c), _d(f), _d(m))
    return f, m


def run(mesh: Mesh, fl: OrcFlow, s: State, max_iter: int, sampling: int = 1, min_residual: float = 0.0,
        min_aerocoeff_error: float = 0.0):
    hist = np.zeros(max(max_iter, 1))
    rp = OrcRunParams(max_iter, sampling, min_residual, min_aerocoeff_error, _d(hist))
    st = OrcRunStats()
    rc = lib().orc_run(C.byref(mesh.c), C.byref(fl), C.byref(s.c), C.byref(rp), C.byref(st))
    if rc != 0:
        raise MemoryError("orc_run allocation failed")
    return st, hist[: st.n_rms].copy()


# ------------------------------------------------------------------ reference checker binary
def ref_available() -> bool:
    return os.path.exists(REF_DRIVER)


def ref_call(mode: str, cfg: str, out: str, *extra: str, timeout: float = 600) -> subprocess.CompletedProcess:
    if not ref_available():
        raise RuntimeError(f"reference checker binary missing: {REF_DRIVER}")
    return subprocess.run([REF_DRIVER, mode, cfg, out, *extra], capture_output=True, text=True, timeout=timeout,
                          check=True)


def ref_mesh_arrays(out: str) -> Dict[str, np.ndarray]:
    """Read the arrays dumped by ``e3d_ref_driver mesh`` into the oracle's mesh dict."""
    meta = dict(line.split() for line in open(os.path.join(out, "meta.txt")).read().strip().splitlines())
    rd = lambda n, t: np.fromfile(os.path.join(out, n), dtype=t)  # noqa: E731
    a = {"n_cells": int(meta["n_elem"]), "n_faces": int(meta["n_face"]), "n_faces_int": int(meta["n_face_int"]),
         "face2cell": rd("face2elem.i32", np.int32), "face_unit_normal": rd("face_unit_normal.f64", np.float64),
         "face_normal": rd("face_normal.f64", np.float64), "face_area": rd("face_area.f64", np.float64),
         "face_center": rd("face_center.f64", np.float64), "cell_volume": rd("cell_volume.f64", np.float64),
         "cell_centroid": rd("cell_centroid.f64", np.float64),
         "cell2face_ptr": rd("elem2face_ptr.i32", np.int32), "cell2face": rd("elem2face.i32", np.int32),
         "cell2cell": rd("elem2elem.i32", np.int32),
         "face2node_ptr": rd("face2node_ptr.i32", np.int32), "face2node": rd("face2node.i32", np.int32)}
    for tag in ("wall", "farfield", "sym"):
        for part in ("ghost", "interior", "face"):
            a[f"{tag}_{part}"] = rd(f"{tag}_{part}.i32", np.int32)
    return a


def ref_state(out: str, prefix: str = "") -> Dict[str, np.ndarray]:
    return {k: np.fromfile(os.path.join(out, f"{prefix}{k}.f64")) for k in STATE_KEYS}
