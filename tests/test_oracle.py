"""The CPU oracle is pinned to the reference solver.

Each golden fixture (tests/golden/*.npz, made by tests/golden/make_golden.py from the unmodified
reference solver) holds the reference's own mesh arrays, one iteration body from a perturbed
state, and a Run() history.  The oracle, fed the reference's arrays, must reproduce every output
bit for bit.  When the reference checker binary is built, the same comparison also runs live on
freshly generated meshes.
"""
import os
import shutil

import numpy as np
import pytest

import pyoracle as po
from cases import CASES, perturbed_state
from euler3d_b200 import meshgen as mg
from euler3d_b200.solver import FlowConfig

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIXTURES = ["channel", "channel_supersonic", "ogrid", "tets", "pyramids"]


def load(name):
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    mesh = {k[len("mesh_"):]: z[k] for k in z.files if k.startswith("mesh_")}
    for k in ("n_cells", "n_faces", "n_faces_int"):
        mesh[k] = int(mesh[k])
    mach, aoa, cfl, gamma = z["flow"]
    return z, po.Mesh(mesh), po.flow(mach, aoa, gamma, cfl)


def assert_bitwise(a, b, what):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, what
    diff = np.flatnonzero(a != b)
    assert diff.size == 0, f"{what}: {diff.size} entries differ (first {diff[:5]})"


@pytest.mark.parametrize("name", FIXTURES)
def test_iteration_body_matches_reference(name):
    z, m, fl = load(name)
    s = po.State(m, {k: z[f"stage_in_{k}"] for k in po.STATE_KEYS})
    po.update_bc(m, fl, s)
    for k in po.STATE_KEYS:
        assert_bitwise(s.a[k], z[f"stage_bc_{k}"], f"ghosts after updateBC ({k})")
    R = po.compute_residual(m, fl, s)
    assert_bitwise(R.ravel(), z["stage_residual"], "computeResidual")
    assert_bitwise(po.time_step(m, fl, s), z["stage_dt"], "TimeStepMethod2")
    R5 = po.runge_kutta(m, fl, s, R)
    assert_bitwise(R5.ravel(), z["stage_residual5"], "stage-5 residual")
    for k in po.STATE_KEYS:
        assert_bitwise(s.a[k], z[f"stage_rk_{k}"], f"state after RungeKutta ({k})")
    assert po.rms(m, R5) == z["stage_rms"][0]


@pytest.mark.parametrize("name", FIXTURES)
def test_run_history_matches_reference(name):
    z, m, fl = load(name)
    s = po.freestream(m, fl)
    st, hist = po.run(m, fl, s, len(z["hist_rms"]))
    assert st.iterations == len(z["hist_rms"])
    assert_bitwise(hist, z["hist_rms"], "density RMS history")
    for k in po.STATE_KEYS:
        assert_bitwise(s.a[k], z[f"hist_final_{k}"], f"final state ({k})")


def test_freestream_is_preserved_on_closed_uniform_box():
    """All-farfield box in uniform flow (the reference's empty-domain example): R is round-off."""
    raw = mg.bump_channel(6, 4, 3, jitter=0.05, seed=9, bump=1e-9)
    for mk in raw.markers:
        mk.tag = "farfield"
    from euler3d_b200.solver import Mesh

    m = po.Mesh(Mesh.from_raw(raw).arrays())
    fl = po.flow(0.5, 3.0, 1.4, 1.0)
    s = po.freestream(m, fl)
    po.update_bc(m, fl, s)
    R = po.compute_residual(m, fl, s)
    assert np.max(np.abs(R)) < 1e-12


@pytest.mark.skipif(not po.ref_available(), reason="reference checker binary not built (make -C oracle ref)")
@pytest.mark.parametrize("seed", [101, 202])
def test_live_against_reference_binary(seed, tmp_path):
    """Fresh meshes and states, compared live with the reference solver."""
    from euler3d_b200.solver import Mesh

    rng = np.random.default_rng(seed)
    raws = [mg.bump_channel(10, 6, 3, seed=seed), mg.biconvex_ogrid(16, 6, 2, seed=seed),
            mg.bump_box_tets(3, seed=seed)]
    for i, raw in enumerate(raws):
        case = mg.CaseConfig(mach=float(rng.uniform(0.3, 1.6)), aoa=float(rng.uniform(-4, 6)),
                             cfl=float(rng.uniform(0.5, 1.5)), max_iter=1)
        d = str(tmp_path / f"c{i}")
        cfg = mg.write_case(raw, case, d)
        po.ref_call("mesh", cfg, d + "/mesh")
        arrays = po.ref_mesh_arrays(d + "/mesh")
        ours = Mesh.read(d + "/mesh.par").arrays()
        for k, v in arrays.items():
            if isinstance(v, np.ndarray):
                assert_bitwise(ours[k], v, f"mesh array {k}")
        m = po.Mesh(arrays)
        fl = po.flow(case.mach, case.aoa, 1.4, case.cfl)
        st = perturbed_state(arrays, FlowConfig(mach=case.mach, aoa=case.aoa, cfl=case.cfl), seed=seed + i)
        sp = d + "/state.f64"
        np.concatenate([st[k] for k in po.STATE_KEYS]).tofile(sp)
        po.ref_call("stage", cfg, d + "/stage", sp)
        s = po.State(m, st)
        po.update_bc(m, fl, s)
        R = po.compute_residual(m, fl, s)
        assert_bitwise(R.ravel(), np.fromfile(d + "/stage/residual.f64"), "residual")
        po.runge_kutta(m, fl, s, R)
        ref_rk = po.ref_state(d + "/stage", "rk_")
        for k in po.STATE_KEYS:
            assert_bitwise(s.a[k], ref_rk[k], f"state after RungeKutta ({k})")
        shutil.rmtree(d, ignore_errors=True)


INTEGRATORS = os.path.join(GOLDEN, "integrators.npz")
# variant -> (integrator (0 RK5, 1 explicit Euler), residual smoothing)
INTEGRATOR_VARIANTS = {"euler": (1, False), "euler_smooth": (1, True), "rk5_smooth": (0, True)}


@pytest.mark.parametrize("name", ["channel", "ogrid", "tets"])
@pytest.mark.parametrize("variant", list(INTEGRATOR_VARIANTS))
def test_integrators_match_reference(name, variant):
    """Explicit Euler (TIME_INTEGRATION= 0) and residual smoothing (RESIDUAL_SMOOTHING= 1), with RK5
    too: the oracle's Run() history and final state equal the reference's bit for bit."""
    g = np.load(INTEGRATORS)
    z, m, _ = load(name)
    mach, aoa, cfl, gamma = z["flow"]
    integ, smooth = INTEGRATOR_VARIANTS[variant]
    fl = po.flow(mach, aoa, gamma, cfl, integrator=integ, smoothing=smooth)
    ref_rms = g[f"{name}__{variant}__rms"]
    s = po.freestream(m, fl)
    st, hist = po.run(m, fl, s, len(ref_rms))
    assert st.iterations == len(ref_rms)
    assert (st.smooth_sweeps > 0) == smooth
    assert_bitwise(hist, ref_rms, "density RMS history")
    for k in po.STATE_KEYS:
        assert_bitwise(s.a[k], g[f"{name}__{variant}__final_{k}"], f"final state ({k})")


def test_smoothing_passes():
    """One Jacobi pass when nothing changes by more than 1e-16, else exactly two (the reference's
    loop ends after its second pass); each pass is R_c = (R0_c + 0.25 sum R_j) / (1 + 0.25 n)."""
    z, m, _ = load("tets")
    R0 = np.random.default_rng(0).standard_normal((m.n_cells, 5))
    Rs, n = po.smooth_residuals(m, R0)
    assert n == 2
    f2c = np.asarray(m.a["face2cell"]).reshape(-1, 2)
    c2f_ptr, c2f = np.asarray(m.a["cell2face_ptr"]), np.asarray(m.a["cell2face"])

    def jacobi(last):
        out = np.empty_like(last)
        for c in range(m.n_cells):
            faces = c2f[c2f_ptr[c]:c2f_ptr[c + 1]]
            nb = [f2c[f][1] if f2c[f][0] == c else f2c[f][0] for f in faces]
            s = np.zeros(5)
            for j in nb:
                if j < m.n_cells:
                    s = s + last[j] * 0.25
            out[c] = (R0[c] + s) / (1 + len(faces) * 0.25)
        return out

    assert np.array_equal(Rs, jacobi(jacobi(R0)))
    Z, n0 = po.smooth_residuals(m, np.zeros((m.n_cells, 5)))
    assert n0 == 1 and not Z.any()
