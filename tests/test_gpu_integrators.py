"""Explicit Euler (TIME_INTEGRATION= 0) and residual smoothing (RESIDUAL_SMOOTHING= 1) on the GPU,
against the oracle (itself pinned bit for bit to the reference, tests/test_oracle.py).

FP64_EXACT must equal the oracle bit for bit for the state and the density RMS (ghost E of
supersonic-outflow ghosts differs in the last bit, at most 1e-13 relative), with the same iteration
counts; FP64 stays within 1e-10 relative per cell."""
import numpy as np
import pytest

import pyoracle as po
from cases import CASES, STATE_KEYS, perturbed_state, prepared
from euler3d_b200 import _lib
from euler3d_b200.batch import Batch
from euler3d_b200.solver import EulerSolver
from test_gpu_parity import FP64_RTOL, RMS_RTOL, assert_state_equal, rel_err

pytestmark = pytest.mark.gpu

# variant -> (integrator, smoothing, iterations)
VARIANTS = {"euler": (_lib.INTEGRATOR_EULER, False, 60), "euler_smooth": (_lib.INTEGRATOR_EULER, True, 40),
            "rk5_smooth": (_lib.INTEGRATOR_RK5, True, 20)}


def setup(name, variant, precision=_lib.PREC_FP64_EXACT, **kw):
    integ, smooth, n = VARIANTS[variant]
    flow = CASES[name].flow(precision=precision, integrator=integ, smoothing=smooth, ordering=_lib.ORDER_SPATIAL, **kw)
    arrays = prepared(name)
    m = po.Mesh(arrays)
    fl = po.flow(flow.mach, flow.aoa, flow.gamma, flow.cfl, flow.sref, flow.cref, flow.ref_point, tuple(flow.cl),
                 tuple(flow.cd), tuple(flow.cm), integrator=integ, smoothing=smooth)
    return arrays, flow, m, fl, n


@pytest.mark.parametrize("name", ["channel", "channel_supersonic", "ogrid", "tets"])
@pytest.mark.parametrize("variant", list(VARIANTS))
@pytest.mark.parametrize("kernel", [_lib.KERNEL_GATHER, _lib.KERNEL_TILE])
def test_exact_matches_oracle(name, variant, kernel):
    arrays, flow, m, fl, n = setup(name, variant)
    o = po.freestream(m, fl)
    ost, ohist = po.run(m, fl, o, n, sampling=3)
    s = EulerSolver(arrays, flow)
    st = s.run(n, sampling=3, stage_kernel=kernel)
    assert st["iterations"] == ost.iterations == n
    assert_state_equal(s.get_state(), o.a, m.n_cells, ghost_E_rtol=1e-13)
    assert rel_err(s.rms_history(), ohist) <= RMS_RTOL
    assert (st["cl"], st["cd"], st["cm"]) == (ost.cl, ost.cd, ost.cm)


@pytest.mark.parametrize("variant", list(VARIANTS))
def test_exact_from_perturbed_state(variant):
    """Every farfield branch (ghost Mach numbers across 1) and smoothing of a rough residual."""
    arrays, flow, m, fl, n = setup("channel_supersonic", variant)
    st0 = perturbed_state(arrays, flow, seed=31)
    o = po.State(m, st0)
    ost, ohist = po.run(m, fl, o, 12)
    s = EulerSolver(arrays, flow)
    s.set_state(st0)
    s.run(12)
    assert_state_equal(s.get_state(), o.a, m.n_cells, ghost_E_rtol=1e-13)
    assert rel_err(s.rms_history(), ohist) <= RMS_RTOL


@pytest.mark.parametrize("name", ["c1", "tets", "ogrid"])
@pytest.mark.parametrize("variant", list(VARIANTS))
def test_fast_within_tolerance(name, variant):
    arrays, flow, m, fl, n = setup(name, variant, precision=_lib.PREC_FP64)
    o = po.freestream(m, fl)
    po.run(m, fl, o, n)
    s = EulerSolver(arrays, flow)
    s.run(n)
    g = s.get_state()
    speed = np.sqrt(o.a["u"] ** 2 + o.a["v"] ** 2 + o.a["w"] ** 2)
    for k in ("rho", "u", "v", "w", "p", "E", "H"):
        scale = speed if k in ("u", "v", "w") else np.abs(o.a[k])
        err = np.max(np.abs(g[k] - o.a[k]) / scale)
        assert err <= FP64_RTOL, (k, err)


def test_euler_convergence_iteration_count():
    """Explicit Euler to a 1e-8 drop of the first RMS takes the oracle's iteration count."""
    arrays, flow, m, fl, _ = setup("channel", "euler")
    o = po.freestream(m, fl)
    _, h0 = po.run(m, fl, o, 1)
    tol = h0[0] * 1e-8
    o = po.freestream(m, fl)
    ost, _ = po.run(m, fl, o, 20000, sampling=50, min_residual=tol)
    assert ost.converged == 1
    for prec in (_lib.PREC_FP64_EXACT, _lib.PREC_FP64):
        s = EulerSolver(arrays, CASES["channel"].flow(precision=prec, integrator=_lib.INTEGRATOR_EULER))
        st = s.run(20000, sampling=50, min_residual=tol, check_every=64)
        assert st["stop_reason"] == _lib.STOP_RESIDUAL
        assert st["iterations"] == ost.iterations, prec
        s2 = EulerSolver(arrays, CASES["channel"].flow(precision=prec, integrator=_lib.INTEGRATOR_EULER))
        st2 = s2.run(20000, sampling=50, min_residual_drop=1e-8, check_every=64)
        assert st2["iterations"] == ost.iterations, prec


@pytest.mark.parametrize("variant", ["euler", "euler_smooth"])
def test_euler_runs_compose(variant):
    """The conservative state explicit Euler carries stays on the device between runs."""
    arrays, flow, _, _, _ = setup("tets", variant)
    a = EulerSolver(arrays, flow)
    a.run(7, check_every=4)
    a.run(6, check_every=2)
    b = EulerSolver(arrays, flow)
    b.run(13)
    ga, gb = a.get_state(), b.get_state()
    for k in STATE_KEYS:
        assert np.array_equal(ga[k], gb[k]), k


def test_smoothing_profile_mode_matches_graphs():
    arrays, flow, _, _, _ = setup("ogrid", "rk5_smooth")
    a = EulerSolver(arrays, flow)
    a.run(6)
    b = EulerSolver(arrays, flow)
    st = b.run(6, profile_stages=True)
    assert st["stage_launches"] == 30 and st["kernel_launches"] == 6 * (5 * 4 + 2)
    for k in STATE_KEYS:
        assert np.array_equal(a.get_state()[k], b.get_state()[k]), k


def test_nonfinite_smoothing_reported():
    arrays, flow, _, _, _ = setup("channel", "euler_smooth", precision=_lib.PREC_FP64)
    st = perturbed_state(arrays, flow, seed=3)
    st["p"][5] = -1.0
    s = EulerSolver(arrays, flow)
    s.set_state(st)
    with pytest.raises(_lib.E3DError) as e:
        s.run(50)
    assert e.value.status == _lib.E3D_ERR_NONFINITE
    s.set_freestream()
    assert s.run(2)["iterations"] == 2


def test_unsupported_combinations_are_refused():
    arrays = prepared("channel")
    with pytest.raises(_lib.E3DError) as e:
        EulerSolver(arrays, CASES["channel"].flow(precision=_lib.PREC_FP32_FLUX, integrator=_lib.INTEGRATOR_EULER))
    assert e.value.status == _lib.E3D_ERR_INVALID_ARG
    with pytest.raises(_lib.E3DError):
        EulerSolver(arrays, CASES["channel"].flow(precision=_lib.PREC_FP32_FLUX, smoothing=True))
    with pytest.raises(_lib.E3DError):
        EulerSolver(arrays, CASES["channel"].flow(integrator=7))
    s = EulerSolver(arrays, CASES["channel"].flow(integrator=_lib.INTEGRATOR_EULER))
    with pytest.raises(_lib.E3DError):
        Batch().add(s, max_iter=10)
    with pytest.raises(_lib.E3DError):
        s.run_noalloc(10)
