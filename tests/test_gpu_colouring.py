"""The face-colouring stage variants (FP64 mode) against the oracle and the face-tile kernel.

Colouring evaluates each face once, one launch per class of faces that share no cell, and adds
F*S to the residuals of its two cells in global memory; a last kernel updates every cell.  A cell
sums its faces in class order rather than in the reference's face order, so the residual differs
from the other FP64 kernels' in the last bits: it is held to 1e-12 of the largest residual of each
component, the time step and the ghost states (per face, the same arithmetic) are compared bit for
bit with the face-tile kernel, and 100 iterations stay within the 1e-10 per-cell bar of the plain
double-precision path.  Two runs give the same bits (the class order is fixed).
"""
import numpy as np
import pytest

import pyoracle as po
from cases import CASES, STATE_KEYS, perturbed_state, prepared
from euler3d_b200 import _lib
from euler3d_b200.solver import EulerSolver
from test_gpu_integrators import VARIANTS, setup
from test_gpu_parity import FP64_RTOL, oracle_setup, rel_err

pytestmark = pytest.mark.gpu

COLOUR = [_lib.KERNEL_COLOUR, _lib.KERNEL_COLOUR_B]
MESHES = ["channel", "channel_supersonic", "ogrid", "tets", "pyramids"]


def max_rel_fields(g, o):
    speed = np.sqrt(o["u"] ** 2 + o["v"] ** 2 + o["w"] ** 2)
    worst = 0.0
    for k in ("rho", "u", "v", "w", "p", "E", "H"):
        scale = speed if k in ("u", "v", "w") else np.abs(o[k])
        worst = max(worst, float(np.max(np.abs(g[k] - o[k]) / scale)))
    return worst


@pytest.mark.parametrize("name", MESHES)
@pytest.mark.parametrize("kernel", COLOUR)
@pytest.mark.parametrize("scheme", [_lib.SCHEME_ROE, _lib.SCHEME_AUSM])
def test_residual(name, kernel, scheme):
    flow = CASES[name].flow(precision=_lib.PREC_FP64, ordering=_lib.ORDER_SPATIAL, scheme=scheme)
    arrays, m, fl = oracle_setup(name, flow)
    st = perturbed_state(arrays, flow, seed=17)
    out = {}
    for k in (kernel, _lib.KERNEL_TILE):
        s = EulerSolver(arrays, flow)
        s.run(0, stage_kernel=k)  # select the variant
        s.set_state(st)
        R, dt = s.residual()
        out[k] = (R, dt, s.get_state())
    R, dt, g = out[kernel]
    Rt, dtt, gt = out[_lib.KERNEL_TILE]
    scale = np.max(np.abs(Rt), axis=0) + 1e-300
    assert np.max(np.abs(R - Rt) / scale) <= 1e-12
    assert np.array_equal(dt, dtt)
    for k in STATE_KEYS:
        assert np.array_equal(g[k], gt[k]), k
    if scheme == _lib.SCHEME_ROE:  # and against the oracle (the reference's residual)
        o = po.State(m, st)
        po.update_bc(m, fl, o)
        Ro = po.compute_residual(m, fl, o)
        scale = np.max(np.abs(Ro), axis=0) + 1e-300
        assert np.max(np.abs(R - Ro) / scale) <= 1e-12


@pytest.mark.parametrize("name", ["c1", "tets", "ogrid"])
@pytest.mark.parametrize("kernel", COLOUR)
def test_100_iterations(name, kernel):
    flow = CASES[name].flow(precision=_lib.PREC_FP64, ordering=_lib.ORDER_SPATIAL)
    arrays, m, fl = oracle_setup(name, flow)
    o = po.freestream(m, fl)
    _, ohist = po.run(m, fl, o, 100)
    s = EulerSolver(arrays, flow)
    st = s.run(100, stage_kernel=kernel)
    assert st["iterations"] == 100
    assert max_rel_fields(s.get_state(), o.a) <= FP64_RTOL
    assert rel_err(s.rms_history(), ohist) <= 1e-8


def test_deterministic():
    name = "ogrid"
    flow = CASES[name].flow(precision=_lib.PREC_FP64, ordering=_lib.ORDER_SPATIAL)
    out = []
    for _ in range(2):
        s = EulerSolver(prepared(name), flow)
        s.run(20, stage_kernel=_lib.KERNEL_COLOUR)
        out.append((s.get_state(), s.rms_history()))
    for k in STATE_KEYS:
        assert np.array_equal(out[0][0][k], out[1][0][k]), k
    assert np.array_equal(out[0][1], out[1][1])


def test_block_sizes_agree():
    """128 and 512 faces per block: the same classes in the same order, the same bits."""
    name = "tets"
    flow = CASES[name].flow(precision=_lib.PREC_FP64, ordering=_lib.ORDER_SPATIAL)
    states = []
    for kernel in COLOUR:
        s = EulerSolver(prepared(name), flow)
        s.run(15, stage_kernel=kernel)
        states.append(s.get_state())
    for k in STATE_KEYS:
        assert np.array_equal(states[0][k], states[1][k]), k


@pytest.mark.parametrize("variant", list(VARIANTS))
def test_with_smoothing_and_euler(variant):
    """Explicit Euler and residual smoothing on the colouring residual, against the oracle."""
    arrays, flow, m, fl, n = setup("tets", variant, precision=_lib.PREC_FP64)
    o = po.freestream(m, fl)
    po.run(m, fl, o, n)
    s = EulerSolver(arrays, flow)
    st = s.run(n, stage_kernel=_lib.KERNEL_COLOUR)
    assert st["iterations"] == n
    assert max_rel_fields(s.get_state(), o.a) <= FP64_RTOL


def test_refused_outside_fp64():
    name = "channel"
    for prec in (_lib.PREC_FP64_EXACT, _lib.PREC_FP32_FLUX):
        s = EulerSolver(prepared(name), CASES[name].flow(precision=prec, ordering=_lib.ORDER_SPATIAL))
        with pytest.raises(_lib.E3DError) as e:
            s.run(1, stage_kernel=_lib.KERNEL_COLOUR)
        assert e.value.status == _lib.E3D_ERR_INVALID_ARG
        assert s.info()["variant_ms"][5] == s.info()["variant_ms"][6] == -1.0


def test_launch_count():
    """One launch per class and the update per stage, plus the RMS and the force integral per
    iteration."""
    name = "tets"
    s = EulerSolver(prepared(name), CASES[name].flow(precision=_lib.PREC_FP64, ordering=_lib.ORDER_SPATIAL))
    st = s.run(4, stage_kernel=_lib.KERNEL_COLOUR, check_every=4)  # one graph of 4 iterations
    per_iter = st["kernel_launches"] / 4
    stages = (per_iter - 2) / 5
    assert per_iter == int(per_iter) and stages == int(stages)
    assert 4 + 1 <= stages <= 7 + 1  # tetrahedra need at least 4 classes and at most 2 x 4 - 1
