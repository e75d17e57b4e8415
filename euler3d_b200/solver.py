"""Python face of the C ABI: prepared meshes and the GPU solver handle.

Names follow the reference solver (src/solver/EulerSolver.cpp, include/solver/FlowField.hpp):
:class:`Mesh` stands for ``Mesh<MeshPartition>`` + ``Metrics``, :class:`EulerSolver` for the
``EulerSolver`` object whose :meth:`EulerSolver.run` replaces ``EulerSolver::Run()``; flow
state dicts hold FlowField's arrays ``rho u v w p E H M`` (interior cells, then ghosts).
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import Dict, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import check

STATE_KEYS = ("rho", "u", "v", "w", "p", "E", "H", "M")
MESH_INT_ARRAYS = ("face2cell", "cell2face_ptr", "cell2face", "cell2cell", "face2node_ptr", "face2node",
                   "wall_ghost", "wall_interior", "wall_face", "farfield_ghost", "farfield_interior",
                   "farfield_face", "sym_ghost", "sym_interior", "sym_face")
MESH_DOUBLE_ARRAYS = ("face_normal", "face_unit_normal", "face_center", "face_area", "cell_volume", "cell_centroid")


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


class Mesh:
    """A mesh prepared by the library: connectivity, metrics and ghost lists in the reference numbering."""

    def write_boundary(self, path: str) -> None:
        """``<partition>.bry`` as the reference's WriteSolution writes it (wall cells and face nodes)."""
        check(_lib.load().e3d_mesh_write_boundary(self._h, path.encode()))

    def __init__(self, handle: C.c_void_p):
        self._h = handle

    @classmethod
    def read(cls, path: str, cref: float = 1.0, threads: int = 0) -> "Mesh":
        lib = _lib.load()
        h = C.c_void_p()
        check(lib.e3d_mesh_read(path.encode(), cref, threads, C.byref(h)))
        return cls(h)

    @classmethod
    def read_partitions(cls, paths: Sequence[str], cref: float = 1.0, threads: int = 0) -> "Mesh":
        """The partition files of a multi-partition case merged into one mesh (e3d_mesh_read_partitions)."""
        lib = _lib.load()
        h = C.c_void_p()
        arr = (C.c_char_p * len(paths))(*[p.encode() for p in paths])
        check(lib.e3d_mesh_read_partitions(arr, len(paths), cref, threads, C.byref(h)))
        return cls(h)

    def partition_cell_ptr(self) -> np.ndarray:
        """First cell of each partition (and the cell count) for a mesh read from partition files."""
        return self.array("partition_cell_ptr")

    @classmethod
    def from_raw(cls, raw, cref: float = 1.0, threads: int = 0) -> "Mesh":
        """Prepare a :class:`euler3d_b200.meshgen.RawMesh` held in memory."""
        lib = _lib.load()
        xyz = np.ascontiguousarray(raw.xyz, np.float64)
        vtk = np.ascontiguousarray(raw.elem_vtk, np.int32)
        eptr, enodes = raw.csr()
        tags = [m.tag.encode() for m in raw.markers]
        tag_arr = (C.c_char_p * max(len(tags), 1))(*tags)
        mptr = np.zeros(len(raw.markers) + 1, np.int32)
        fptr_parts, fn_parts = [], []
        nf = 0
        for i, m in enumerate(raw.markers):
            cnt = np.where(m.vtk == 5, 3, 4).astype(np.int64)
            nodes = m.nodes[np.arange(4)[None, :] < cnt[:, None]]
            fptr_parts.append(cnt)
            fn_parts.append(nodes)
            nf += m.vtk.shape[0]
            mptr[i + 1] = nf
        counts = np.concatenate(fptr_parts) if fptr_parts else np.zeros(0, np.int64)
        fptr = np.zeros(counts.size + 1, np.int64)
        np.cumsum(counts, out=fptr[1:])
        fptr = fptr.astype(np.int32)
        fnodes = (np.concatenate(fn_parts) if fn_parts else np.zeros(0)).astype(np.int32)
        h = C.c_void_p()
        check(lib.e3d_mesh_from_arrays(xyz.shape[0], _dp(xyz), vtk.shape[0], _ip(vtk), _ip(eptr), _ip(enodes),
                                       len(tags), tag_arr, _ip(mptr), _ip(fptr), _ip(fnodes), cref, threads,
                                       C.byref(h)))
        return cls(h)

    def close(self) -> None:
        if self._h:
            _lib.load().e3d_mesh_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> Dict[str, int]:
        i = _lib.MeshInfo()
        check(_lib.load().e3d_mesh_info_get(self._h, C.byref(i)))
        return {k: getattr(i, k) for k, _ in _lib.MeshInfo._fields_}

    def array(self, name: str) -> np.ndarray:
        data, count, is_double = C.c_void_p(), C.c_int64(), C.c_int32()
        check(_lib.load().e3d_mesh_array(self._h, name.encode(), C.byref(data), C.byref(count), C.byref(is_double)))
        n = count.value
        if n == 0:
            return np.zeros(0, np.float64 if is_double.value else np.int32)
        ctype = C.c_double if is_double.value else C.c_int32
        return np.ctypeslib.as_array(C.cast(data, C.POINTER(ctype)), shape=(n,)).copy()

    def arrays(self) -> Dict[str, object]:
        """All prepared arrays plus sizes, in the dict layout the solver descriptor takes."""
        info = self.info()
        d: Dict[str, object] = {"n_cells": info["n_cells"], "n_faces": info["n_faces"],
                                "n_faces_int": info["n_faces_int"]}
        for n in MESH_INT_ARRAYS + MESH_DOUBLE_ARRAYS:
            d[n] = self.array(n)
        return d


class _Desc:
    """An e3d_mesh_desc over numpy arrays (kept alive by this object)."""

    def __init__(self, a: Dict[str, object]):
        keep = {}

        def arr(name, dtype):
            v = np.ascontiguousarray(a.get(name, np.zeros(0)), dtype=dtype)
            if v.size == 0:
                v = np.zeros(1, dtype)
            keep[name] = v
            return v

        d = _lib.MeshDesc()
        d.n_cells, d.n_faces, d.n_faces_int = int(a["n_cells"]), int(a["n_faces"]), int(a["n_faces_int"])
        d.face2cell = _ip(arr("face2cell", np.int32))
        for n in ("face_unit_normal", "face_normal", "face_area", "face_center", "cell_volume"):
            setattr(d, n, _dp(arr(n, np.float64)))
        d.cell2face_ptr = _ip(arr("cell2face_ptr", np.int32))
        d.cell2face = _ip(arr("cell2face", np.int32))
        for tag in ("wall", "farfield", "sym"):
            setattr(d, f"n_{tag}", int(np.asarray(a.get(f"{tag}_ghost", np.zeros(0))).size))
            for part in ("ghost", "interior", "face"):
                setattr(d, f"{tag}_{part}", _ip(arr(f"{tag}_{part}", np.int32)))
        self.keep = keep
        self.c = d


@dataclasses.dataclass
class FlowConfig:
    """The flow / solver keys of an ``.e3d`` file that the hot path consumes."""
    mach: float = 0.5
    aoa: float = 0.0
    gamma: float = 1.4
    cfl: float = 1.5
    sref: float = 1.0
    cref: float = 1.0
    ref_point: Sequence[float] = (0.25, 0.0, 0.0)
    cl: Sequence[int] = (1, 1)      # (axis, sign): MESH_ORIENTATION_CL
    cd: Sequence[int] = (0, 1)
    cm: Sequence[int] = (2, 1)
    scheme: int = _lib.SCHEME_ROE
    precision: int = _lib.PREC_FP64
    ordering: int = _lib.ORDER_NATIVE
    device: int = 0
    integrator: int = _lib.INTEGRATOR_RK5   # TIME_INTEGRATION= 2 (RK5) or 0 (INTEGRATOR_EULER)
    smoothing: bool = False                  # RESIDUAL_SMOOTHING=

    @staticmethod
    def orientation(cl_code: int, cd_code: int):
        """(axis, sign) pairs of SimConfig (src/parser/SimConfig.cpp:185-231) from MESH_ORIENTATION codes."""
        table = [(0, 1), (0, -1), (1, 1), (1, -1), (2, 1), (2, -1)]
        cl, cd = table[cl_code], table[cd_code]
        cm = (3 - cl[0] - cd[0], -cl[1] * cd[1])
        return cl, cd, cm


def run_params(max_iter: int, sampling: int = 1, min_residual: float = 0.0, min_aerocoeff_error: float = 0.0,
               check_every: int = 0, profile_stages: int = 0, stage_kernel: int = 0,
               min_residual_drop: float = 0.0, stall_window: int = 0, stall_below: float = 0.0) -> _lib.RunParams:
    """``e3d_run_params``: MAX_ITER, SAMPLING, MIN_RESIDUAL, MIN_AEROCOEFF_ERROR of the reference's
    config plus the launch options and the relative residual-drop stop.  ``profile_stages``: 0 CUDA
    graphs; 1 (or True) direct launches, every stage kernel timed; 2 CUDA graphs with every stage
    kernel timed by events captured in the graph."""
    return _lib.RunParams(max_iter, sampling, min_residual, min_aerocoeff_error, check_every, int(profile_stages),
                          stage_kernel, min_residual_drop, stall_window, stall_below)


def stats_dict(st: _lib.RunStats) -> Dict[str, object]:
    return {"iterations": st.iterations, "stop_reason": st.stop_reason, "n_rms": st.n_rms,
            "last_rms": st.last_rms, "cl": st.cl, "cd": st.cd, "cm": st.cm, "force": list(st.force),
            "moment": list(st.moment), "device_ms": st.device_ms, "kernel_launches": st.kernel_launches,
            "stage_ms": st.stage_ms, "stage_launches": st.stage_launches}


class EulerSolver:
    """GPU replacement of the reference's ``EulerSolver`` (include/solver/EulerSolver.hpp:89-223)."""

    def __init__(self, mesh, flow: FlowConfig, stream: Optional[int] = None, autotune: bool = True):
        lib = _lib.load()
        arrays = mesh.arrays() if isinstance(mesh, Mesh) else mesh
        self._desc = _Desc(arrays)
        self.n_cells = int(arrays["n_cells"])
        self.flow = flow
        p = _lib.FlowParams()
        p.gamma, p.mach, p.aoa_deg, p.cfl = flow.gamma, flow.mach, flow.aoa, flow.cfl
        p.sref, p.cref = flow.sref, flow.cref
        p.ref_point[:] = list(flow.ref_point)
        p.cl_axis, p.cl_sign = flow.cl
        p.cd_axis, p.cd_sign = flow.cd
        p.cm_axis, p.cm_sign = flow.cm
        p.scheme, p.precision, p.ordering, p.device = flow.scheme, flow.precision, flow.ordering, flow.device
        p.stream = stream
        p.no_autotune = 0 if autotune else 1
        p.integrator, p.residual_smoothing = flow.integrator, int(bool(flow.smoothing))
        h = C.c_void_p()
        check(lib.e3d_solver_create(C.byref(self._desc.c), C.byref(p), C.byref(h)))
        self._h = h
        self.state_size = int(lib.e3d_solver_state_size(h))

    def close(self) -> None:
        if getattr(self, "_h", None):
            _lib.load().e3d_solver_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> Dict[str, object]:
        i = _lib.SolverInfo()
        check(_lib.load().e3d_solver_info_get(self._h, C.byref(i)))
        return {"n_cells": i.n_cells, "n_ghosts": i.n_ghosts, "n_faces": i.n_faces,
                "stage_variant": i.stage_variant, "variant_ms": list(i.variant_ms)[: i.n_variants],
                "tile_smem_bytes": i.tile_smem_bytes,
                "device_bytes": i.device_bytes}

    # ---- state
    def set_state(self, state: Dict[str, np.ndarray]) -> None:
        arrs = [np.ascontiguousarray(state[k], np.float64) for k in STATE_KEYS]
        for a in arrs:
            if a.size != self.state_size:
                raise ValueError(f"state arrays must have {self.state_size} entries")
        ptrs = (C.POINTER(C.c_double) * 8)(*[_dp(a) for a in arrs])
        check(_lib.load().e3d_solver_set_state(self._h, ptrs))

    def set_freestream(self) -> None:
        check(_lib.load().e3d_solver_set_freestream(self._h))

    def get_state(self, out: Optional[Dict[str, np.ndarray]] = None) -> Dict[str, np.ndarray]:
        out = out or {k: np.empty(self.state_size) for k in STATE_KEYS}
        ptrs = (C.POINTER(C.c_double) * 8)(*[_dp(out[k]) for k in STATE_KEYS])
        check(_lib.load().e3d_solver_get_state(self._h, ptrs))
        return out

    # ---- hot path
    def run(self, max_iter: int, sampling: int = 1, min_residual: float = 0.0, min_aerocoeff_error: float = 0.0,
            check_every: int = 0, profile_stages: int = 0, stage_kernel: int = 0,
            min_residual_drop: float = 0.0, stall_window: int = 0, stall_below: float = 0.0) -> Dict[str, object]:
        rp = run_params(max_iter, sampling, min_residual, min_aerocoeff_error, check_every, profile_stages,
                        stage_kernel, min_residual_drop, stall_window, stall_below)
        st = _lib.RunStats()
        status = _lib.load().e3d_solver_run(self._h, C.byref(rp), C.byref(st))
        stats = stats_dict(st)
        try:
            check(status)
        except _lib.E3DError as e:
            e.stats = stats  # how far the run got (a non-finite stop, a timeout)
            raise
        return stats

    def run_noalloc(self, max_iter: int, sampling: int = 1, min_residual: float = 0.0,
                    min_aerocoeff_error: float = 0.0, check_every: int = 0):
        """``e3d_solver_run_noalloc``: the same iterations as :meth:`run` without any device allocation
        (scratch in a fixed 1.5 MiB device array; at most 65,536 iterations per call).  Returns
        (stats, density RMS of every iteration); the handle's own RMS history and coefficient samples
        then report no entries."""
        rp = run_params(max_iter, sampling, min_residual, min_aerocoeff_error, check_every)
        st = _lib.RunStats()
        hist = np.zeros(max(max_iter, 1))
        status = _lib.load().e3d_solver_run_noalloc(self._h, C.byref(rp), C.byref(st), _dp(hist), hist.size)
        check(status)
        stats = stats_dict(st)
        del stats["stage_ms"], stats["stage_launches"]
        return stats, hist[: st.n_rms].copy()

    def set_wait_limit(self, polls: int) -> None:
        """``e3d_solver_set_wait_limit``: polls of the stage kernels' bounded data waits (negative:
        the default).  0 makes every wait give up at once, which exercises the timeout path."""
        check(_lib.load().e3d_solver_set_wait_limit(self._h, polls))

    def rms_history(self) -> np.ndarray:
        n = C.c_int32()
        check(_lib.load().e3d_solver_rms_history(self._h, None, 0, C.byref(n)))
        out = np.zeros(max(n.value, 1))
        check(_lib.load().e3d_solver_rms_history(self._h, _dp(out), n.value, C.byref(n)))
        return out[: n.value]

    def residual(self):
        """(R [n_cells, 5], dt [n_cells]) of updateBC + computeResidual + updateDeltaTime at the current state."""
        R = np.empty(5 * self.n_cells)
        dt = np.empty(self.n_cells)
        check(_lib.load().e3d_solver_residual(self._h, _dp(R), _dp(dt)))
        return R.reshape(-1, 5), dt

    def coefficients(self):
        f, m = np.empty(3), np.empty(3)
        check(_lib.load().e3d_solver_coefficients(self._h, _dp(f), _dp(m)))
        return f, m

    # ---- the reference's output files (byte for byte)
    def coefficient_history(self) -> np.ndarray:
        """[n, 7]: iteration, force (3), moment (3) of every sample of the last run."""
        n = C.c_int32()
        check(_lib.load().e3d_solver_coefficient_history(self._h, None, 0, C.byref(n)))
        out = np.zeros((max(n.value, 1), 7))
        check(_lib.load().e3d_solver_coefficient_history(self._h, _dp(out), n.value, C.byref(n)))
        return out[: n.value]

    def wall_cp(self) -> np.ndarray:
        n = C.c_int32()
        check(_lib.load().e3d_solver_wall_cp(self._h, None, 0, C.byref(n)))
        out = np.zeros(max(n.value, 1))
        check(_lib.load().e3d_solver_wall_cp(self._h, _dp(out), n.value, C.byref(n)))
        return out[: n.value]

    def write_outputs(self, output_dir: str, partition_file: Optional[str] = None, solver_ms: int = 0,
                      total_ms: int = 0, n_cores: int = 1, rank: int = 0) -> None:
        """residuals.dat, cp_part_<rank>.dat and summary.txt into ``output_dir`` and, given the
        partition file name, ``<partition_file>.sol`` (src/Solver.cpp:58-67 writes the same set)."""
        import os

        lib = _lib.load()
        check(lib.e3d_solver_write_residuals(self._h, os.path.join(output_dir, "residuals.dat").encode()))
        check(lib.e3d_solver_write_summary(self._h, os.path.join(output_dir, "summary.txt").encode(), solver_ms,
                                           total_ms, n_cores))
        check(lib.e3d_solver_write_cp(self._h, os.path.join(output_dir, f"cp_part_{rank}.dat").encode()))
        if partition_file:
            check(lib.e3d_solver_write_solution(self._h, (partition_file + ".sol").encode()))
