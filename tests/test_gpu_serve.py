"""Served solves (continuous batching): every request's result is the one it gets alone, whatever
else shares the device and whenever it is admitted; the plain one-at-a-time path agrees with it."""
import numpy as np
import pytest

from cases import STATE_KEYS
from euler3d_b200 import _lib, serve
from euler3d_b200.solver import EulerSolver

pytestmark = pytest.mark.gpu


def stream():
    return serve.request_stream(10, rate=200.0, cells=(800, 6000), seed=7, drops=(1e-6, 1e-8),
                                schemes=(_lib.SCHEME_ROE, _lib.SCHEME_AUSM))


def solo(req, precision=_lib.PREC_FP64):
    s = EulerSolver(serve._prepare(req), serve.request_flow(req, precision), autotune=False)
    st = s.run(200_000, sampling=1_000_000, min_residual_drop=req.drop, stage_kernel=_lib.KERNEL_TILE)
    return st, s.get_state(), serve.final_coefficients(s)


def test_served_equals_alone_with_admission_limits():
    reqs = stream()
    states = {}
    srv = serve.Server(max_members=3, iterations_per_step=24,
                       hbm_budget=3 * serve.footprint_estimate(6000, 20000, _lib.PREC_FP64))
    res = srv.serve(reqs, on_result=lambda r, s: states.__setitem__(r.rid, s.get_state()))
    assert sorted(r.rid for r in res) == list(range(len(reqs)))
    assert srv.peak_members <= 3
    assert any(r.admitted > r.arrival + 1e-3 for r in res)  # some waited for a slot
    for r in res:
        req = reqs[r.rid]
        st, state, coeffs = solo(req)
        assert r.status == _lib.E3D_OK and r.stop_reason == _lib.STOP_RESIDUAL
        assert r.iterations == st["iterations"], r.rid
        assert (r.cl, r.cd, r.cm) == coeffs, r.rid
        for k in STATE_KEYS:
            assert np.array_equal(states[r.rid][k], state[k]), (r.rid, k)
        assert r.latency >= r.finished - r.admitted >= 0


def test_plain_path_agrees():
    reqs = stream()[:5]
    served = {r.rid: r for r in serve.Server(iterations_per_step=16).serve(reqs)}
    plain = {r.rid: r for r in serve.serve_plain(reqs)}
    for rid, p in plain.items():
        s = served[rid]
        assert p.status == _lib.E3D_OK and p.stop_reason == _lib.STOP_RESIDUAL
        assert abs(p.iterations - s.iterations) <= 2, rid
        for a, b in ((p.cl, s.cl), (p.cd, s.cd)):
            assert abs(a - b) <= 1e-8 * max(abs(b), 1e-3), rid
    summ = serve.summarize(list(plain.values()))
    assert summ["solves"] == 5 and summ["p99_latency_s"] >= summ["p50_latency_s"] > 0


@pytest.mark.parametrize("precision", [_lib.PREC_FP64, _lib.PREC_FP32_FLUX])
def test_footprint_estimate_bounds_device_bytes(precision):
    for req in serve.request_stream(6, 0.0, cells=(500, 60000), seed=2):
        arrays = serve._prepare(req)
        s = EulerSolver(arrays, serve.request_flow(req, precision), autotune=False)
        actual = s.info()["device_bytes"]
        est = serve.footprint_estimate(int(arrays["n_cells"]), int(arrays["n_faces"]), precision)
        assert actual <= est <= 3 * actual + (2 << 20), (req.family, arrays["n_cells"], actual, est)


def test_oversized_request_is_refused():
    req = serve.request_stream(1, 0.0, cells=(2000, 2001), seed=1)
    res = serve.Server(hbm_budget=1e5).serve(req)
    assert len(res) == 1 and res[0].status == _lib.E3D_ERR_OOM


def test_precision_ladder():
    """FP32 flux first, FP64 from the FP32 floor to the tolerance: the same outcome as the plain FP64
    solve, lift and drag within 1e-4 relative -- both stop at the same residual, from different
    histories, so they agree as far as that residual converges the forces."""
    reqs = stream()[:6]
    lad = {r.rid: r for r in serve.Server(ladder=True, iterations_per_step=16, stall_window=100).serve(reqs)}
    for req in reqs:
        st, _, coeffs = solo(req)
        r = lad[req.rid]
        assert r.status == _lib.E3D_OK and r.stop_reason == st["stop_reason"] == _lib.STOP_RESIDUAL
        assert r.fp32_iterations > 0
        for a, b in zip((r.cl, r.cd), coeffs[:2]):
            # relative to the coefficient scale: a near-zero lift is not a relative-error measure
            assert abs(a - b) <= 1e-4 * max(abs(b), 1e-2), (req.rid, a, b)


def test_stall_stop():
    """An FP32 solve held to an unreachable tolerance stops on the stall test, not at max_iter."""
    req = stream()[0]
    s = EulerSolver(serve._prepare(req), serve.request_flow(req, _lib.PREC_FP32_FLUX), autotune=False)
    st = s.run(100_000, sampling=1_000_000, min_residual_drop=1e-14, stall_window=100)
    assert st["stop_reason"] == _lib.STOP_STALL and st["iterations"] < 100_000
    h = s.rms_history()
    assert np.min(h[-100:]) >= np.min(h[:-100])  # no new minimum in the last window
