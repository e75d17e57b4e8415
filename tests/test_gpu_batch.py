"""Batches (e3d_batch_*): several solvers of uneven sizes, schemes and flow conditions advanced in
shared launches must each compute exactly what the solver computes alone with the face-tile
kernel -- the same state bit for bit, the same RMS history, iteration count, stop reason and
coefficients -- whatever else is in the batch and whenever members join or leave.  The tolerance
is zero: members share launches but no arithmetic."""
import numpy as np
import pytest

import pyoracle as po
from cases import CASES, STATE_KEYS, perturbed_state, prepared
from euler3d_b200 import _lib
from euler3d_b200 import meshgen as mg
from euler3d_b200.batch import Batch
from euler3d_b200.solver import EulerSolver, FlowConfig, Mesh

pytestmark = pytest.mark.gpu

PRECISIONS = [_lib.PREC_FP64_EXACT, _lib.PREC_FP64, _lib.PREC_FP32_FLUX]
STAT_KEYS = ("iterations", "stop_reason", "n_rms", "last_rms", "cl", "cd", "cm", "force", "moment")

# (case, scheme, initial state seed or None for the freestream, run parameters)
MIX = [
    ("channel", _lib.SCHEME_ROE, None, dict(max_iter=300, sampling=5, min_residual_drop=1e-3)),
    ("channel_supersonic", _lib.SCHEME_AUSM, 21, dict(max_iter=90, sampling=3)),
    ("ogrid", _lib.SCHEME_ROE, 22, dict(max_iter=120, sampling=4, min_aerocoeff_error=1e-3)),
    ("tets", _lib.SCHEME_AUSM, None, dict(max_iter=70, sampling=1)),
    ("c1", _lib.SCHEME_ROE, None, dict(max_iter=150, sampling=10, min_residual_drop=1e-2)),
]


def make_solver(name, scheme, seed, precision):
    arrays = prepared(name)
    flow = CASES[name].flow(precision=precision, scheme=scheme, ordering=_lib.ORDER_SPATIAL)
    s = EulerSolver(arrays, flow)
    if seed is not None:
        s.set_state(perturbed_state(arrays, flow, seed=seed))
    return s


def alone(name, scheme, seed, precision, rp):
    s = make_solver(name, scheme, seed, precision)
    stats = s.run(rp["max_iter"], sampling=rp.get("sampling", 1), min_residual=rp.get("min_residual", 0.0),
                  min_aerocoeff_error=rp.get("min_aerocoeff_error", 0.0),
                  min_residual_drop=rp.get("min_residual_drop", 0.0), stage_kernel=_lib.KERNEL_TILE)
    return s.get_state(), s.rms_history(), stats


def assert_same(result, ref, label):
    state, hist, stats = result
    rstate, rhist, rstats = ref
    for k in STATE_KEYS:
        diff = np.flatnonzero(state[k] != rstate[k])
        assert diff.size == 0, f"{label} {k}: {diff.size} entries differ"
    assert np.array_equal(hist, rhist), label
    for k in STAT_KEYS:
        assert stats[k] == rstats[k], (label, k, stats[k], rstats[k])


def collect(solver, stats):
    return solver.get_state(), solver.rms_history(), stats


@pytest.mark.parametrize("precision,kernel", [(p, _lib.BATCH_KERNEL_TILES) for p in PRECISIONS] +
                         [(p, _lib.BATCH_KERNEL_WS) for p in PRECISIONS])
def test_mix_equals_alone(precision, kernel):
    refs = [alone(n, sc, sd, precision, rp) for n, sc, sd, rp in MIX]
    b = Batch()
    b.set_kernel(kernel)
    solvers = []
    for n, sc, sd, rp in MIX:
        s = make_solver(n, sc, sd, precision)
        b.add(s, **rp)
        solvers.append(s)
    done = b.run_all(iterations_per_step=16)
    assert len(done) == len(MIX)
    by_id = {id(s): (st, status) for s, st, status in done}
    for (n, sc, sd, rp), s, ref in zip(MIX, solvers, refs):
        st, status = by_id[id(s)]
        assert status == _lib.E3D_OK
        assert_same(collect(s, st), ref, n)
    # the members stopped for different reasons at different iterations
    assert len({by_id[id(s)][0]["iterations"] for s in solvers}) > 2
    b.close()


@pytest.mark.parametrize("precision,kernel", [(_lib.PREC_FP64, _lib.BATCH_KERNEL_TILES),
                                              (_lib.PREC_FP32_FLUX, _lib.BATCH_KERNEL_TILES),
                                              (_lib.PREC_FP64, _lib.BATCH_KERNEL_WS),
                                              (_lib.PREC_FP32_FLUX, _lib.BATCH_KERNEL_WS)])
def test_staggered_admission(precision, kernel):
    """Members join a running batch between steps (continuous admission) and leave as they stop."""
    refs = [alone(n, sc, sd, precision, rp) for n, sc, sd, rp in MIX]
    b = Batch()
    b.set_kernel(kernel)
    solvers, results = [], {}
    for i, (n, sc, sd, rp) in enumerate(MIX):
        s = make_solver(n, sc, sd, precision)
        b.add(s, **rp)
        solvers.append(s)
        b.step(6 + 4 * i)
        for r, st, status in b.retire():
            assert status == _lib.E3D_OK
            results[id(r)] = collect(r, st)
    for r, st, status in b.run_all(10):
        results[id(r)] = collect(r, st)
    for (n, *_), s, ref in zip(MIX, solvers, refs):
        assert_same(results[id(s)], ref, n)


def test_exact_member_matches_oracle():
    """Anchor to the oracle: an FP64_EXACT member in a mix equals the CPU restatement bit for bit."""
    name = "ogrid"
    flow = CASES[name].flow(precision=_lib.PREC_FP64_EXACT)
    arrays = prepared(name)
    m = po.Mesh(arrays)
    fl = po.flow(flow.mach, flow.aoa, flow.gamma, flow.cfl, flow.sref, flow.cref, flow.ref_point,
                 tuple(flow.cl), tuple(flow.cd), tuple(flow.cm))
    o = po.freestream(m, fl)
    ost, ohist = po.run(m, fl, o, 40, sampling=4)
    b = Batch()
    s = EulerSolver(arrays, flow)
    b.add(s, max_iter=40, sampling=4)
    others = [make_solver("tets", _lib.SCHEME_AUSM, 5, _lib.PREC_FP64_EXACT),
              make_solver("c1", _lib.SCHEME_ROE, None, _lib.PREC_FP64_EXACT)]
    for x in others:
        b.add(x, max_iter=25)
    done = {id(r): st for r, st, _ in b.run_all(8)}
    g = s.get_state()
    for k in STATE_KEYS:
        n = m.n_cells if k == "E" else g[k].size  # ghost E differs from the oracle by summation order
        assert np.array_equal(g[k][:n], o.a[k][:n]), k
    assert done[id(s)]["iterations"] == ost.iterations
    assert (done[id(s)]["cl"], done[id(s)]["cd"]) == (ost.cl, ost.cd)
    assert np.array_equal(s.rms_history(), ohist)  # summed in the reference's order in FP64_EXACT


def test_many_members_capacity_growth():
    """More members than the initial table capacity (graph rebuilt for the larger tables), each a
    different flow condition on its own mesh."""
    rng = np.random.default_rng(3)
    specs = []
    for i in range(12):
        nx = int(rng.integers(8, 24))
        specs.append((mg.bump_channel(nx, max(4, nx // 2), 2, seed=i), float(rng.uniform(0.3, 0.8)),
                      float(rng.uniform(-4, 6)), int(i % 2)))
    refs, solvers = [], []
    b = Batch()
    for raw, mach, aoa, scheme in specs:
        arrays = Mesh.from_raw(raw).arrays()
        flow = FlowConfig(mach=mach, aoa=aoa, cfl=1.2, scheme=scheme, precision=_lib.PREC_FP64)
        a = EulerSolver(arrays, flow)
        st = a.run(60, sampling=6, min_residual_drop=1e-2, stage_kernel=_lib.KERNEL_TILE)
        refs.append((a.get_state(), a.rms_history(), st))
        s = EulerSolver(arrays, flow)
        b.add(s, max_iter=60, sampling=6, min_residual_drop=1e-2)
        solvers.append(s)
    info = b.info()
    assert info["n_members"] == 12 and info["n_running"] == 12
    got = {id(r): collect(r, st) for r, st, _ in b.run_all(12)}
    for s, ref in zip(solvers, refs):
        assert_same(got[id(s)], ref, "member")
    assert b.info()["n_members"] == 0


def test_retired_solver_is_usable_again():
    """A retired member continues alone exactly as if it had run alone throughout."""
    name = "tets"
    ref = make_solver(name, _lib.SCHEME_ROE, 4, _lib.PREC_FP64)
    ref.run(30, stage_kernel=_lib.KERNEL_TILE)
    ref.run(20, stage_kernel=_lib.KERNEL_TILE)
    b = Batch()
    s = make_solver(name, _lib.SCHEME_ROE, 4, _lib.PREC_FP64)
    b.add(s, max_iter=30)
    b.add(make_solver("channel", _lib.SCHEME_ROE, None, _lib.PREC_FP64), max_iter=100)
    b.step(30)
    retired = b.retire()
    assert [r for r, _, _ in retired] == [s]
    s.run(20, stage_kernel=_lib.KERNEL_TILE)
    g, r = s.get_state(), ref.get_state()
    for k in STATE_KEYS:
        assert np.array_equal(g[k], r[k]), k
    b.close()


def test_membership_rules():
    b = Batch()
    s = make_solver("channel", _lib.SCHEME_ROE, None, _lib.PREC_FP64)
    b.add(s, max_iter=10)
    with pytest.raises(_lib.E3DError) as e:
        s.set_freestream()
    assert e.value.status == _lib.E3D_ERR_INVALID_ARG
    with pytest.raises(_lib.E3DError):
        s.run(2)
    with pytest.raises(_lib.E3DError):
        b.add(s, max_iter=10)  # already a member
    other = Batch()
    with pytest.raises(_lib.E3DError):
        other.add(s, max_iter=10)  # member of another batch
    with pytest.raises(_lib.E3DError):
        b.add(make_solver("channel", _lib.SCHEME_ROE, None, _lib.PREC_FP32_FLUX), max_iter=10)  # precision
    x = make_solver("tets", _lib.SCHEME_ROE, None, _lib.PREC_FP64)
    with pytest.raises(_lib.E3DError):
        b.remove(x)  # not a member
    # removing a running member hands it back at an iteration boundary
    b.add(x, max_iter=100)
    b.step(4)
    st = b.remove(x)
    assert st["iterations"] == 4 and st["n_rms"] == 4
    x.run(1)
    # destroying a member's solver takes it out of the batch
    y = make_solver("tets", _lib.SCHEME_ROE, None, _lib.PREC_FP64)
    b.add(y, max_iter=100)
    b._members.pop(y._h.value)
    y.close()
    assert b.info()["n_members"] == 1
    assert b.step(10) == 0
    assert [r for r, _, _ in b.retire()] == [s]
    s.set_freestream()


def test_zero_iterations_and_empty_batch():
    b = Batch()
    assert b.step(4) == 0
    s = make_solver("channel", _lib.SCHEME_ROE, None, _lib.PREC_FP64)
    b.add(s, max_iter=0)
    assert b.info()["n_running"] == 0
    (r, st, status), = b.retire()
    assert r is s and st["iterations"] == 0 and status == _lib.E3D_OK


def test_nonfinite_member_reported_others_unaffected():
    """A member that blows up stops with E3D_ERR_NONFINITE; the others finish as they would alone."""
    prec = _lib.PREC_FP64
    ref = alone("ogrid", _lib.SCHEME_ROE, 22, prec, dict(max_iter=60, sampling=4))
    arrays = prepared("channel")
    flow = CASES["channel"].flow(precision=prec)
    bad_state = perturbed_state(arrays, flow, seed=3)
    bad_state["p"][5] = -1.0
    bad = EulerSolver(arrays, flow)
    bad.set_state(bad_state)
    good = make_solver("ogrid", _lib.SCHEME_ROE, 22, prec)
    b = Batch()
    b.add(bad, max_iter=60)
    b.add(good, max_iter=60, sampling=4)
    res = {id(r): (r, st, status) for r, st, status in b.run_all(8)}
    assert res[id(bad)][2] == _lib.E3D_ERR_NONFINITE
    assert res[id(good)][2] == _lib.E3D_OK
    assert_same(collect(good, res[id(good)][1]), ref, "good")
    bad.set_freestream()
    assert bad.run(2)["iterations"] == 2
