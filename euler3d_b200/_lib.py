"""ctypes binding of ``libeuler3d_b200.so`` (declarations: include/euler3d_b200.h).

There is no fallback: if the shared library is missing or cannot be loaded this module raises,
and every solver call runs the CUDA path or fails with the library's status and message.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libeuler3d_b200.so")

ABI_VERSION = 3
E3D_OK, E3D_ERR_INVALID_ARG, E3D_ERR_OOM, E3D_ERR_NONFINITE, E3D_ERR_TIMEOUT, E3D_ERR_CUDA, E3D_ERR_MESH = range(7)
SCHEME_ROE, SCHEME_AUSM = 0, 1
PREC_FP64_EXACT, PREC_FP64, PREC_FP32_FLUX = 0, 1, 2
ORDER_NATIVE, ORDER_RCM, ORDER_SPATIAL = 0, 1, 2
KERNEL_AUTO, KERNEL_GATHER, KERNEL_GATHER_B, KERNEL_TILE, KERNEL_TILE_PIPE, KERNEL_TILE_B3 = 0, 1, 2, 3, 4, 5
KERNEL_COLOUR, KERNEL_COLOUR_B = 6, 7  # face colouring, 128 / 512 faces per block (FP64)
STOP_MAX_ITER, STOP_RESIDUAL, STOP_COEFFICIENTS, STOP_STALL = 0, 1, 2, 3
INTEGRATOR_RK5, INTEGRATOR_EULER = 0, 1
BATCH_KERNEL_TILES, BATCH_KERNEL_WS = 0, 1

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class MeshDesc(C.Structure):
    _fields_ = [("n_cells", C.c_int32), ("n_faces", C.c_int32), ("n_faces_int", C.c_int32),
                ("face2cell", _ip), ("face_unit_normal", _dp), ("face_normal", _dp), ("face_area", _dp),
                ("face_center", _dp), ("cell_volume", _dp), ("cell2face_ptr", _ip), ("cell2face", _ip),
                ("n_wall", C.c_int32), ("wall_ghost", _ip), ("wall_interior", _ip), ("wall_face", _ip),
                ("n_farfield", C.c_int32), ("farfield_ghost", _ip), ("farfield_interior", _ip),
                ("farfield_face", _ip),
                ("n_sym", C.c_int32), ("sym_ghost", _ip), ("sym_interior", _ip), ("sym_face", _ip)]


class MeshInfo(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("n_cells", "n_faces", "n_faces_int", "n_nodes", "n_wall", "n_farfield",
                                         "n_sym")]


class FlowParams(C.Structure):
    _fields_ = [("gamma", C.c_double), ("mach", C.c_double), ("aoa_deg", C.c_double), ("cfl", C.c_double),
                ("sref", C.c_double), ("cref", C.c_double), ("ref_point", C.c_double * 3),
                ("cl_axis", C.c_int32), ("cl_sign", C.c_int32), ("cd_axis", C.c_int32), ("cd_sign", C.c_int32),
                ("cm_axis", C.c_int32), ("cm_sign", C.c_int32), ("scheme", C.c_int32), ("precision", C.c_int32),
                ("ordering", C.c_int32), ("device", C.c_int32), ("stream", C.c_void_p),
                ("no_autotune", C.c_int32), ("integrator", C.c_int32), ("residual_smoothing", C.c_int32)]


class RunParams(C.Structure):
    _fields_ = [("max_iter", C.c_int32), ("sampling", C.c_int32), ("min_residual", C.c_double),
                ("min_aerocoeff_error", C.c_double), ("check_every", C.c_int32), ("profile_stages", C.c_int32),
                ("stage_kernel", C.c_int32), ("min_residual_drop", C.c_double), ("stall_window", C.c_int32),
                ("stall_below", C.c_double)]


class RunStats(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("stop_reason", C.c_int32), ("n_rms", C.c_int32),
                ("last_rms", C.c_double), ("cl", C.c_double), ("cd", C.c_double), ("cm", C.c_double),
                ("force", C.c_double * 3), ("moment", C.c_double * 3), ("device_ms", C.c_double),
                ("kernel_launches", C.c_int64), ("stage_ms", C.c_double), ("stage_launches", C.c_int64)]


class SolverInfo(C.Structure):
    _fields_ = [("n_cells", C.c_int32), ("n_ghosts", C.c_int32), ("n_faces", C.c_int32),
                ("stage_variant", C.c_int32), ("n_variants", C.c_int32), ("variant_ms", C.c_float * 8),
                ("tile_smem_bytes", C.c_int32), ("device_bytes", C.c_int64)]


class BatchInfo(C.Structure):
    _fields_ = [("n_members", C.c_int32), ("n_running", C.c_int32), ("n_tiles", C.c_int32),
                ("graph_builds", C.c_int32), ("member_device_bytes", C.c_int64), ("device_bytes", C.c_int64),
                ("last_step_ms", C.c_double), ("kernel_launches", C.c_int64)]


class E3DError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{message} (status {status})")
        self.status = status


# Every symbol include/euler3d_b200.h declares, with its ctypes signature.
SIGNATURES = {
    "e3d_mesh_read": (C.c_int, [C.c_char_p, C.c_double, C.c_int32, C.POINTER(C.c_void_p)]),
    "e3d_mesh_from_arrays": (C.c_int, [C.c_int32, _dp, C.c_int32, _ip, _ip, _ip, C.c_int32,
                                       C.POINTER(C.c_char_p), _ip, _ip, _ip, C.c_double, C.c_int32,
                                       C.POINTER(C.c_void_p)]),
    "e3d_mesh_info_get": (C.c_int, [C.c_void_p, C.POINTER(MeshInfo)]),
    "e3d_mesh_array": (C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(C.c_void_p), C.POINTER(C.c_int64),
                                 C.POINTER(C.c_int32)]),
    "e3d_mesh_destroy": (None, [C.c_void_p]),
    "e3d_mesh_describe": (C.c_int, [C.c_void_p, C.POINTER(MeshDesc)]),
    "e3d_solver_create": (C.c_int, [C.POINTER(MeshDesc), C.POINTER(FlowParams), C.POINTER(C.c_void_p)]),
    "e3d_solver_destroy": (None, [C.c_void_p]),
    "e3d_solver_state_size": (C.c_int64, [C.c_void_p]),
    "e3d_solver_info_get": (C.c_int, [C.c_void_p, C.POINTER(SolverInfo)]),
    "e3d_solver_set_state": (C.c_int, [C.c_void_p, C.POINTER(_dp)]),
    "e3d_solver_get_state": (C.c_int, [C.c_void_p, C.POINTER(_dp)]),
    "e3d_solver_set_freestream": (C.c_int, [C.c_void_p]),
    "e3d_solver_run": (C.c_int, [C.c_void_p, C.POINTER(RunParams), C.POINTER(RunStats)]),
    "e3d_solver_rms_history": (C.c_int, [C.c_void_p, _dp, C.c_int32, C.POINTER(C.c_int32)]),
    "e3d_solver_run_noalloc": (C.c_int, [C.c_void_p, C.POINTER(RunParams), C.POINTER(RunStats), _dp, C.c_int32]),
    "e3d_solver_set_wait_limit": (C.c_int, [C.c_void_p, C.c_int32]),
    "e3d_fast_reciprocals": (C.c_int, [C.c_int32, _dp, C.c_int64, _dp]),
    "e3d_solver_residual": (C.c_int, [C.c_void_p, _dp, _dp]),
    "e3d_solver_coefficients": (C.c_int, [C.c_void_p, _dp, _dp]),
    "e3d_solver_coefficient_history": (C.c_int, [C.c_void_p, _dp, C.c_int32, C.POINTER(C.c_int32)]),
    "e3d_solver_wall_cp": (C.c_int, [C.c_void_p, _dp, C.c_int32, C.POINTER(C.c_int32)]),
    "e3d_solver_write_residuals": (C.c_int, [C.c_void_p, C.c_char_p]),
    "e3d_solver_write_cp": (C.c_int, [C.c_void_p, C.c_char_p]),
    "e3d_solver_write_solution": (C.c_int, [C.c_void_p, C.c_char_p]),
    "e3d_solver_write_summary": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int64, C.c_int64, C.c_int32]),
    "e3d_mesh_write_boundary": (C.c_int, [C.c_void_p, C.c_char_p]),
    "e3d_mesh_read_partitions": (C.c_int, [C.POINTER(C.c_char_p), C.c_int32, C.c_double, C.c_int32,
                                           C.POINTER(C.c_void_p)]),
    "e3d_batch_create": (C.c_int, [C.c_int32, C.c_void_p, C.POINTER(C.c_void_p)]),
    "e3d_batch_set_kernel": (C.c_int, [C.c_void_p, C.c_int32]),
    "e3d_batch_destroy": (None, [C.c_void_p]),
    "e3d_batch_add": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(RunParams)]),
    "e3d_batch_step": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32)]),
    "e3d_batch_retire": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(RunStats), C.POINTER(C.c_int),
                                   C.c_int32, C.POINTER(C.c_int32)]),
    "e3d_batch_remove": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(RunStats)]),
    "e3d_batch_info_get": (C.c_int, [C.c_void_p, C.POINTER(BatchInfo)]),
    "e3d_status_string": (C.c_char_p, [C.c_int]),
    "e3d_last_error": (C.c_char_p, []),
    "e3d_abi_version": (C.c_int32, []),
}

_lib = None


def load() -> C.CDLL:
    """Load the CUDA library; raises if it is missing (build it with ``python -m euler3d_b200.build``)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"euler3d_b200 CUDA library not built: {LIB_PATH} is missing "
                          "(run `python -m euler3d_b200.build`)")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.e3d_abi_version() != ABI_VERSION:
        raise ImportError("euler3d_b200 library ABI version mismatch")
    _lib = lib
    return lib


def check(status: int) -> None:
    if status != E3D_OK:
        lib = load()
        raise E3DError(status, lib.e3d_last_error().decode(errors="replace") or
                       lib.e3d_status_string(status).decode())
