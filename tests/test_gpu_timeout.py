"""The device timeout path, exercised without a GPU fault.

Every wait of the face-tile stage kernels on their data barrier is bounded.  When a wait gives up,
the kernel lets the copies it issued land (again bounded), sets the run's fault word and returns
without touching its cells; the RMS kernel that follows stops the run, the host reports
E3D_ERR_TIMEOUT, and the CUDA context and the solver stay usable.  The reference has no device
waits (its loop, src/solver/EulerSolver.cpp:84-159, has no failure exit at all), so this is the
library's own failure detection.

A wait is made to run out by the solver's test hook ``e3d_solver_set_wait_limit(solver, 0)``: the
first poll of every barrier is skipped, so every wait gives up at once while the copies it waits
for still complete normally.  Nothing here can hang or fault: the drain after the give-up keeps the
full poll limit, and every copy it waits for was issued and lands.
"""
import numpy as np
import pytest

import pyoracle as po
from cases import CASES, STATE_KEYS, perturbed_state, prepared
from euler3d_b200 import _lib
from euler3d_b200.batch import Batch
from euler3d_b200.solver import EulerSolver

pytestmark = pytest.mark.gpu

# (precision, stage kernel) pairs with bounded waits: face tiles, the warp-specialised persistent
# kernel and face tiles at seven (FP64) or eight (FP32_FLUX) blocks per SM
WAITING_KERNELS = [
    (_lib.PREC_FP64_EXACT, _lib.KERNEL_TILE),
    (_lib.PREC_FP64_EXACT, _lib.KERNEL_TILE_PIPE),
    (_lib.PREC_FP64, _lib.KERNEL_TILE_B3),
    (_lib.PREC_FP32_FLUX, _lib.KERNEL_TILE_PIPE),
    (_lib.PREC_FP32_FLUX, _lib.KERNEL_TILE_B3),
]


def oracle_rk(name, flow, state, iters):
    arrays = prepared(name)
    m = po.Mesh(arrays)
    fl = po.flow(flow.mach, flow.aoa, flow.gamma, flow.cfl, flow.sref, flow.cref, flow.ref_point,
                 tuple(flow.cl), tuple(flow.cd), tuple(flow.cm))
    o = po.State(m, state)
    po.run(m, fl, o, iters)
    return o.a, m.n_cells


@pytest.mark.parametrize("precision,kernel", WAITING_KERNELS)
def test_timeout_stops_run_and_solver_recovers(precision, kernel):
    name = "channel"
    flow = CASES[name].flow(precision=precision, ordering=_lib.ORDER_SPATIAL)
    arrays = prepared(name)
    st = perturbed_state(arrays, flow, seed=31)
    s = EulerSolver(arrays, flow)
    s.set_state(st)
    s.set_wait_limit(0)
    with pytest.raises(_lib.E3DError) as e:
        s.run(20, stage_kernel=kernel)
    assert e.value.status == _lib.E3D_ERR_TIMEOUT
    # the run stopped in its first iteration: no RMS was computed, no iteration counted
    assert e.value.stats["iterations"] == 0 and e.value.stats["n_rms"] == 0
    # the handle and the context stay usable: with the default limit the same solver runs a normal
    # iteration from a freshly loaded state (FP64_EXACT: the oracle's bits)
    s.set_wait_limit(-1)
    s.set_state(st)
    stats = s.run(1, stage_kernel=kernel)
    assert stats["iterations"] == 1
    g = s.get_state()
    if precision == _lib.PREC_FP64_EXACT:
        o, n = oracle_rk(name, flow, st, 1)
        for k in STATE_KEYS:
            if k == "E":  # supersonic-outflow ghost E is recomputed from H (round-off, see test_gpu_parity)
                assert np.array_equal(g[k][:n], o[k][:n])
            else:
                assert np.array_equal(g[k], o[k]), k
    else:
        ref = EulerSolver(arrays, flow)
        ref.set_state(st)
        ref.run(1, stage_kernel=kernel)
        r = ref.get_state()
        for k in STATE_KEYS:
            assert np.array_equal(g[k], r[k]), k


@pytest.mark.parametrize("precision,kernel", [(_lib.PREC_FP64, _lib.BATCH_KERNEL_TILES),
                                              (_lib.PREC_FP32_FLUX, _lib.BATCH_KERNEL_TILES),
                                              (_lib.PREC_FP64, _lib.BATCH_KERNEL_WS),
                                              (_lib.PREC_FP32_FLUX, _lib.BATCH_KERNEL_WS)])
def test_timeout_in_batch_member(precision, kernel):
    """A member whose waits give up is retired with E3D_ERR_TIMEOUT; the member beside it is not
    disturbed (it equals its run alone bit for bit), and the timed-out solver runs normally once
    it is handed back."""
    bad_name, good_name = "channel", "tets"
    bad_flow = CASES[bad_name].flow(precision=precision, ordering=_lib.ORDER_SPATIAL)
    good_flow = CASES[good_name].flow(precision=precision, ordering=_lib.ORDER_SPATIAL)
    bad = EulerSolver(prepared(bad_name), bad_flow)
    good = EulerSolver(prepared(good_name), good_flow)
    alone = EulerSolver(prepared(good_name), good_flow)
    alone_stats = alone.run(40, sampling=4, stage_kernel=_lib.KERNEL_TILE)
    bad.set_wait_limit(0)
    b = Batch()
    b.set_kernel(kernel)
    b.add(bad, 40, sampling=4)
    b.add(good, 40, sampling=4)
    done = {id(s): (stats, status) for s, stats, status in b.run_all(8)}
    b.close()
    stats, status = done[id(bad)]
    assert status == _lib.E3D_ERR_TIMEOUT and stats["iterations"] == 0
    stats, status = done[id(good)]
    assert status == _lib.E3D_OK
    assert stats["iterations"] == alone_stats["iterations"] == 40
    assert np.array_equal(good.rms_history(), alone.rms_history())
    g, a = good.get_state(), alone.get_state()
    for k in STATE_KEYS:
        assert np.array_equal(g[k], a[k]), k
    bad.set_wait_limit(-1)
    bad.set_freestream()
    assert bad.run(3)["iterations"] == 3


def test_wait_limit_hook_rules():
    name = "channel"
    s = EulerSolver(prepared(name), CASES[name].flow())
    s.set_wait_limit(1 << 30)  # clamped to the default; a normal run
    assert s.run(2)["iterations"] == 2
    b = Batch()
    b.add(s, 4)
    with pytest.raises(_lib.E3DError) as e:
        s.set_wait_limit(0)
    assert e.value.status == _lib.E3D_ERR_INVALID_ARG
    b.close()
