"""Parity at the sizes that are benchmarked.

The other parity tests run meshes of a few hundred to a few thousand cells.  These run the
configurations the measurements are quoted on, so that anything that depends on size -- 32-bit
offsets, tiles whose halo nears the 1024-local-cell encoding, the Morton tiles of a real bump, the
RMS reductions over 10^5 blocks -- is compared with the oracle where it is timed:

* the transonic biconvex O-grid, 256 x 128 x 4 hexahedra split into 262,144 prisms (Mach 0.8,
  AoA 1.25, CFL 1.2), Roe and AUSM: FP64_EXACT equals the oracle bit for bit after 5 iterations
  from the freestream, FP64 within 1e-10;
* the 64^3 x 6 = 1,572,864-tetrahedron bump box: FP64_EXACT equals the oracle bit for bit after
  3 iterations, and FP64 stays within 1e-10 of FP64_EXACT after 50 iterations;
* the 128^3 x 6 = 12,582,912-tetrahedron bump box of the bench: one RK5 iteration from the
  freestream, FP64_EXACT bit for bit and FP64 within 1e-10 of the oracle.

Tolerances: bit for bit in FP64_EXACT (ghost E of supersonic-outflow ghosts, recomputed from H at
later stages, within 1e-13); 1e-10 relative per cell for FP64, velocity components relative to the
local flow speed -- the bar the plain double-precision path is held to.
"""
import numpy as np
import pytest

import pyoracle as po
from cases import STATE_KEYS
from euler3d_b200 import _lib
from euler3d_b200 import meshgen as mg
from euler3d_b200.solver import EulerSolver, FlowConfig, Mesh

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-10
GHOST_E_RTOL = 1e-13


def oracle_of(arrays, flow):
    m = po.Mesh(arrays)
    fl = po.flow(flow.mach, flow.aoa, flow.gamma, flow.cfl, flow.sref, flow.cref, flow.ref_point,
                 tuple(flow.cl), tuple(flow.cd), tuple(flow.cm), scheme=flow.scheme)
    return m, fl


def assert_bitwise(g, o, n):
    for k in STATE_KEYS:
        if k == "E":
            assert np.array_equal(g[k][:n], o[k][:n]), k
            rel = np.abs(g[k][n:] - o[k][n:]) / np.abs(o[k][n:])
            assert rel.size == 0 or rel.max() <= GHOST_E_RTOL, k
        else:
            diff = np.flatnonzero(g[k] != o[k])
            assert diff.size == 0, f"{k}: {diff.size} entries differ, first {diff[:5]}"


def max_rel(g, o, n):
    """Largest per-cell relative difference over the interior fields (velocity components
    relative to the local flow speed)."""
    speed = np.sqrt(o["u"][:n] ** 2 + o["v"][:n] ** 2 + o["w"][:n] ** 2)
    worst = 0.0
    for k in ("rho", "u", "v", "w", "p", "E", "H"):
        scale = speed if k in ("u", "v", "w") else np.abs(o[k][:n])
        worst = max(worst, float(np.max(np.abs(g[k][:n] - o[k][:n]) / scale)))
    return worst


_meshes = {}


def mesh(name):
    if name not in _meshes:
        raw = {"c2": lambda: mg.biconvex_ogrid(256, 128, 4),
               "tets64": lambda: mg.bump_box_tets(64),
               "tets128": lambda: mg.bump_box_tets(128)}[name]()
        _meshes.clear()  # one large mesh held at a time
        _meshes[name] = Mesh.from_raw(raw).arrays()
    return _meshes[name]


@pytest.mark.parametrize("scheme", [_lib.SCHEME_ROE, _lib.SCHEME_AUSM])
def test_c2_ogrid_5_iterations(scheme):
    arrays = mesh("c2")
    assert int(arrays["n_cells"]) == 262_144
    flow = FlowConfig(mach=0.8, aoa=1.25, cfl=1.2, scheme=scheme, precision=_lib.PREC_FP64_EXACT,
                      ordering=_lib.ORDER_SPATIAL)
    m, fl = oracle_of(arrays, flow)
    o = po.freestream(m, fl)
    _, ohist = po.run(m, fl, o, 5)
    s = EulerSolver(arrays, flow)
    assert s.run(5)["iterations"] == 5
    assert_bitwise(s.get_state(), o.a, m.n_cells)
    assert np.array_equal(s.rms_history(), ohist)
    fast = EulerSolver(arrays, FlowConfig(mach=0.8, aoa=1.25, cfl=1.2, scheme=scheme, precision=_lib.PREC_FP64,
                                          ordering=_lib.ORDER_SPATIAL))
    fast.run(5)
    assert max_rel(fast.get_state(), o.a, m.n_cells) <= FP64_RTOL


def test_tets64_exact_and_fp64():
    arrays = mesh("tets64")
    assert int(arrays["n_cells"]) == 64 ** 3 * 6
    exact_flow = FlowConfig(mach=0.6, aoa=0.0, cfl=1.0, precision=_lib.PREC_FP64_EXACT, ordering=_lib.ORDER_SPATIAL)
    m, fl = oracle_of(arrays, exact_flow)
    o = po.freestream(m, fl)
    _, ohist = po.run(m, fl, o, 3)
    exact = EulerSolver(arrays, exact_flow)
    exact.run(3)
    assert_bitwise(exact.get_state(), o.a, m.n_cells)
    assert np.array_equal(exact.rms_history(), ohist)
    # 47 more iterations: FP64 against FP64_EXACT after 50
    exact.run(47)
    fast = EulerSolver(arrays, FlowConfig(mach=0.6, aoa=0.0, cfl=1.0, precision=_lib.PREC_FP64,
                                          ordering=_lib.ORDER_SPATIAL))
    fast.run(50)
    e = exact.get_state()
    assert max_rel(fast.get_state(), e, m.n_cells) <= FP64_RTOL


def test_bench_mesh_one_iteration():
    """The bench's 12,582,912-tetrahedron mesh: one RK5 iteration from the freestream."""
    arrays = mesh("tets128")
    n = int(arrays["n_cells"])
    assert n == 128 ** 3 * 6
    exact_flow = FlowConfig(mach=0.6, aoa=0.0, cfl=1.0, precision=_lib.PREC_FP64_EXACT, ordering=_lib.ORDER_SPATIAL)
    m, fl = oracle_of(arrays, exact_flow)
    o = po.freestream(m, fl)
    _, ohist = po.run(m, fl, o, 1)
    exact = EulerSolver(arrays, exact_flow, autotune=False)
    exact.run(1)
    assert_bitwise(exact.get_state(), o.a, n)
    assert np.array_equal(exact.rms_history(), ohist)
    exact.close()
    fast = EulerSolver(arrays, FlowConfig(mach=0.6, aoa=0.0, cfl=1.0, precision=_lib.PREC_FP64,
                                          ordering=_lib.ORDER_SPATIAL))
    fast.run(1)
    assert max_rel(fast.get_state(), o.a, n) <= FP64_RTOL
