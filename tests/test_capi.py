"""The C ABI library: it loads, exports every function include/euler3d_b200.h declares, and reports
argument errors with a status and a message (no GPU needed)."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from cases import prepared
from euler3d_b200 import _lib
from euler3d_b200.solver import EulerSolver, FlowConfig

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "euler3d_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(e3d_[a-z0-9_]+)\s*\(", text)))


def test_header_and_binding_agree():
    assert set(declared_functions()) == set(_lib.SIGNATURES)


def test_library_exports_every_declared_symbol():
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True, check=True)
    exported = set(re.findall(r"\bT (e3d_\w+)", out.stdout))
    missing = set(declared_functions()) - exported
    assert not missing, missing
    lib = _lib.load()
    for name in declared_functions():
        assert hasattr(lib, name)


def test_version_and_status_strings():
    lib = _lib.load()
    assert lib.e3d_abi_version() == _lib.ABI_VERSION == 3
    assert lib.e3d_status_string(_lib.E3D_ERR_NONFINITE) == b"non-finite solution"


def test_null_arguments_are_rejected():
    lib = _lib.load()
    h = C.c_void_p()
    assert lib.e3d_solver_create(None, None, C.byref(h)) == _lib.E3D_ERR_INVALID_ARG
    assert b"NULL" in lib.e3d_last_error()
    assert lib.e3d_solver_run(None, None, None) == _lib.E3D_ERR_INVALID_ARG
    assert lib.e3d_mesh_read(None, 1.0, 0, C.byref(h)) == _lib.E3D_ERR_INVALID_ARG
    n = C.c_int32()
    assert lib.e3d_batch_create(0, None, None) == _lib.E3D_ERR_INVALID_ARG
    assert lib.e3d_batch_add(None, None, None) == _lib.E3D_ERR_INVALID_ARG
    assert lib.e3d_batch_step(None, 2, C.byref(n)) == _lib.E3D_ERR_INVALID_ARG
    assert lib.e3d_batch_retire(None, None, None, None, 0, C.byref(n)) == _lib.E3D_ERR_INVALID_ARG
    assert lib.e3d_batch_remove(None, None, None) == _lib.E3D_ERR_INVALID_ARG
    assert lib.e3d_batch_info_get(None, None) == _lib.E3D_ERR_INVALID_ARG
    lib.e3d_batch_destroy(None)


def test_batch_refuses_without_gpu():
    """No sm_100 device: creating a batch fails with a CUDA status instead of running elsewhere."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    assert _lib.load().e3d_batch_create(0, None, C.byref(h)) in (_lib.E3D_ERR_CUDA, _lib.E3D_ERR_INVALID_ARG)
    assert not h.value


def test_descriptor_validation():
    a = dict(prepared("channel"))
    bad = dict(a)
    bad["face2cell"] = a["face2cell"].copy()
    bad["face2cell"][1] = a["n_cells"] + 10**6  # right cell of an interior face out of range
    with pytest.raises(_lib.E3DError) as e:
        EulerSolver(bad, FlowConfig())
    assert e.value.status in (_lib.E3D_ERR_INVALID_ARG, _lib.E3D_ERR_CUDA)
    with pytest.raises(_lib.E3DError) as e:
        EulerSolver(a, FlowConfig(gamma=0.9))
    assert e.value.status == _lib.E3D_ERR_INVALID_ARG


def test_no_silent_cpu_path():
    """Without an sm_100 GPU the solver refuses to run instead of falling back to the CPU."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(_lib.E3DError) as e:
        EulerSolver(prepared("channel"), FlowConfig())
    assert e.value.status == _lib.E3D_ERR_CUDA


def test_mesh_arrays_roundtrip():
    a = prepared("tets")
    n = a["n_cells"]
    assert a["cell2face_ptr"][-1] == 4 * n
    assert np.all(a["cell_volume"] > 0)
