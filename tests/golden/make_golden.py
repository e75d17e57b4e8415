"""Generate the golden fixtures of tests/golden/ by running the reference solver itself.

Needs the reference checker binary (``make -C oracle ref``, built from the reference sources).
For each small seeded case it stores, as one compressed .npz:

* the reference's own mesh arrays (connectivity, metrics, ghost lists) -- the input of the oracle
  and the expected output of the product's mesh preparation;
* one iteration body from a perturbed flow state (``e3d_ref_driver stage``): ghost states after
  updateBC, residual, time step, stage-5 residual, state after RungeKutta, density RMS;
* ``n_hist`` iterations of Run() from the freestream (``e3d_ref_driver history``): the density RMS
  of every iteration and the final state.

``integrators.npz`` holds Run() histories of three cases under the other time-integration settings
(TIME_INTEGRATION= 0 explicit Euler, with and without RESIDUAL_SMOOTHING= 1, and RK5 with residual
smoothing): the density RMS of every iteration and the final state.

``outputs/<run>/`` holds the files the reference's own writers produce for two short runs of the
bump channel (``e3d_ref_driver outputs``, timings fixed at 1234 / 5678 ms): residuals.dat,
cp_part_0.dat, summary.txt, mesh.par.sol and mesh.par.bry, with the run's settings in run.json.

``reference_partitions.npz`` holds the bytes of the reference's partitioned test case
(test/mesh/StructuredBlock_8_p0..3.par) and of the mesh it was cut from.

Run from the repository root:  python tests/golden/make_golden.py [integrators | outputs | partitions | case <name>...]
"""
import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.dirname(HERE))

import pyoracle as po  # noqa: E402
from cases import CASES, perturbed_state  # noqa: E402
from euler3d_b200 import meshgen as mg  # noqa: E402

GOLDEN_CASES = {"channel": 40, "channel_supersonic": 30, "ogrid": 30, "tets": 30, "pyramids": 30}
# (TIME_INTEGRATION=, RESIDUAL_SMOOTHING=, iterations) per variant, for these cases
INTEGRATOR_VARIANTS = {"euler": (0, 0, 30), "euler_smooth": (0, 1, 20), "rk5_smooth": (2, 1, 10)}
INTEGRATOR_CASES = ("channel", "ogrid", "tets")
REFERENCE_TEST_MESHES = ("StructuredBlock_8.su2", "naca0012_9x9x5_unittest_mesh.su2", "stackedCubes.su2",
                         "stackedTetrahedron.su2")


def case_config(case, time_integration=2, residual_smoothing=0):
    return mg.CaseConfig(mach=case.mach, aoa=case.aoa, cfl=case.cfl, max_iter=1, sampling=1,
                         orientation_cl=2, orientation_cd=0, ref_point=(0.25, 0.0, 0.0),
                         time_integration=time_integration, residual_smoothing=residual_smoothing)


def write_state(path, st):
    np.concatenate([st[k] for k in po.STATE_KEYS]).astype(np.float64).tofile(path)


def make_case(name, n_hist, work):
    case = CASES[name]
    raw = case.raw()
    d = os.path.join(work, name)
    cfg = mg.write_case(raw, case_config(case), d)
    po.ref_call("mesh", cfg, os.path.join(d, "mesh"))
    mesh = po.ref_mesh_arrays(os.path.join(d, "mesh"))
    out = {f"mesh_{k}": np.asarray(v) for k, v in mesh.items()}
    # the mesh itself, as the product's preparation reads it
    eptr, enodes = raw.csr()
    out.update(raw_xyz=raw.xyz, raw_elem_vtk=raw.elem_vtk, raw_elem_ptr=eptr, raw_elem_nodes=enodes,
               raw_marker_tags=np.array([m.tag for m in raw.markers]),
               raw_marker_sizes=np.array([m.vtk.size for m in raw.markers]),
               raw_marker_nodes=np.concatenate([m.nodes for m in raw.markers]))
    # one iteration body from a perturbed state
    from euler3d_b200.solver import FlowConfig  # noqa: E402

    flow = FlowConfig(mach=case.mach, aoa=case.aoa, cfl=case.cfl)
    st = perturbed_state(mesh, flow, seed=21)
    sp = os.path.join(d, "state.f64")
    write_state(sp, st)
    po.ref_call("stage", cfg, os.path.join(d, "stage"), sp)
    sd = os.path.join(d, "stage")
    for k in po.STATE_KEYS:
        out[f"stage_in_{k}"] = st[k]
        out[f"stage_bc_{k}"] = np.fromfile(os.path.join(sd, f"bc_{k}.f64"))
        out[f"stage_rk_{k}"] = np.fromfile(os.path.join(sd, f"rk_{k}.f64"))
    out["stage_residual"] = np.fromfile(os.path.join(sd, "residual.f64"))
    out["stage_dt"] = np.fromfile(os.path.join(sd, "dt.f64"))
    out["stage_residual5"] = np.fromfile(os.path.join(sd, "residual_stage5.f64"))
    out["stage_rms"] = np.fromfile(os.path.join(sd, "rms.f64"))
    # Run() history from the freestream
    po.ref_call("history", cfg, os.path.join(d, "hist"), str(n_hist))
    hd = os.path.join(d, "hist")
    out["hist_rms"] = np.fromfile(os.path.join(hd, "rms.f64"))
    for k in po.STATE_KEYS:
        out[f"hist_final_{k}"] = np.fromfile(os.path.join(hd, f"{k}.f64"))
    out["flow"] = np.array([case.mach, case.aoa, case.cfl, 1.4])
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    return sum(v.nbytes for v in out.values())


def make_integrators(work):
    out = {}
    for name in INTEGRATOR_CASES:
        case = CASES[name]
        raw = case.raw()
        for var, (ti, rs, n) in INTEGRATOR_VARIANTS.items():
            d = os.path.join(work, f"{name}_{var}")
            cfg = mg.write_case(raw, case_config(case, ti, rs), d)
            po.ref_call("history", cfg, os.path.join(d, "hist"), str(n))
            hd = os.path.join(d, "hist")
            out[f"{name}__{var}__rms"] = np.fromfile(os.path.join(hd, "rms.f64"))
            for k in po.STATE_KEYS:
                out[f"{name}__{var}__final_{k}"] = np.fromfile(os.path.join(hd, f"{k}.f64"))
    np.savez_compressed(os.path.join(HERE, "integrators.npz"), **out)
    return sum(v.nbytes for v in out.values())


# run name -> (case, TIME_INTEGRATION=, MAX_ITER=, SAMPLING=, MIN_RESIDUAL as a fraction of the first RMS)
OUTPUT_RUNS = {"rk5_max_iter": ("channel", 2, 25, 4, 0.0), "euler_residual_exit": ("channel", 0, 400, 7, 1e-2)}


def make_outputs(work):
    import json

    for run, (name, ti, max_iter, sampling, drop) in OUTPUT_RUNS.items():
        case = CASES[name]
        min_res = 0.0
        if drop:  # the absolute MIN_RESIDUAL: a fraction of the first iteration's RMS
            d0 = os.path.join(work, run + "_first")
            cfg0 = mg.write_case(case.raw(), case_config(case, ti), d0)
            po.ref_call("history", cfg0, os.path.join(d0, "hist"), "1")
            min_res = float(np.fromfile(os.path.join(d0, "hist", "rms.f64"))[0]) * drop
        d = os.path.join(work, run)
        cfg = mg.CaseConfig(mach=case.mach, aoa=case.aoa, cfl=case.cfl, max_iter=max_iter, sampling=sampling,
                            min_residual=min_res, orientation_cl=2, orientation_cd=0, ref_point=(0.25, 0.0, 0.0),
                            time_integration=ti)
        cfg_path = mg.write_case(case.raw(), cfg, d)
        po.ref_call("outputs", cfg_path, os.path.join(d, "o"), "1234", "5678")
        dst = os.path.join(HERE, "outputs", run)
        os.makedirs(dst, exist_ok=True)
        for src in ("output/residuals.dat", "output/cp_part_0.dat", "output/summary.txt", "mesh.par.sol",
                    "mesh.par.bry"):
            shutil.copy(os.path.join(d, src), os.path.join(dst, os.path.basename(src)))
        with open(os.path.join(dst, "run.json"), "w") as f:
            json.dump({"case": name, "time_integration": ti, "max_iter": max_iter, "sampling": sampling,
                       "min_residual": min_res, "solver_ms": 1234, "total_ms": 5678}, f, indent=1)


def make_reference_partitions(reference_root):
    """The reference's own partitioned test case (test/mesh/StructuredBlock_8_p0..3.par, written by its
    partitioner) and the mesh it was cut from, as file bytes."""
    out = {}
    d = os.path.join(reference_root, "test", "mesh")
    for f in ["StructuredBlock_8.su2"] + [f"StructuredBlock_8_p{i}.par" for i in range(4)]:
        out[f.replace(".", "_")] = np.frombuffer(open(os.path.join(d, f), "rb").read(), dtype=np.uint8)
    np.savez_compressed(os.path.join(HERE, "reference_partitions.npz"), **out)


def make_reference_meshes(work, reference_root):
    out = {}
    for f in REFERENCE_TEST_MESHES:
        d = os.path.join(work, "refmesh_" + f.split(".")[0])
        os.makedirs(os.path.join(d, "output"), exist_ok=True)
        txt = open(os.path.join(reference_root, "test", "mesh", f)).read()
        par = os.path.join(d, "mesh.par")
        with open(par, "w") as fh:
            fh.write(txt.rstrip("\n") + "\nNINTERNAL_MARKER= 0\n")
        cfg = os.path.join(d, "case.e3d")
        mg.write_e3d(mg.CaseConfig(), cfg, par, os.path.join(d, "output", "out.dat"))
        po.ref_call("mesh", cfg, os.path.join(d, "mesh"), timeout=120)
        key = f.split(".")[0]
        out[f"{key}__par"] = np.frombuffer(open(par, "rb").read(), dtype=np.uint8)
        for k, v in po.ref_mesh_arrays(os.path.join(d, "mesh")).items():
            out[f"{key}__{k}"] = np.asarray(v)
    np.savez_compressed(os.path.join(HERE, "reference_test_meshes.npz"), **out)


def reference_root() -> str:
    """The reference's source tree, from the E3D_REFERENCE_ROOT environment variable (required)."""
    root = os.environ.get("E3D_REFERENCE_ROOT")
    if not root:
        raise SystemExit("set E3D_REFERENCE_ROOT to the reference's source tree")
    return root


def main():
    if not po.ref_available():
        sys.exit("reference checker binary missing: run `make -C oracle ref` first")
    work = tempfile.mkdtemp(prefix="e3dgold")
    try:
        if sys.argv[1:] == ["integrators"]:
            print("integrators", make_integrators(work), "bytes")
            return
        if sys.argv[1:] == ["outputs"]:
            make_outputs(work)
            return
        if sys.argv[1:2] == ["case"]:  # one solver-path fixture: make_golden.py case <name>
            for name in sys.argv[2:]:
                print(name, make_case(name, GOLDEN_CASES[name], work), "bytes")
            return
        if sys.argv[1:] == ["partitions"]:
            make_reference_partitions(reference_root())
            return
        make_outputs(work)
        print("integrators", make_integrators(work), "bytes")
        for name, n in GOLDEN_CASES.items():
            print(name, make_case(name, n, work), "bytes")
        ref_root = reference_root()
        if os.path.isdir(os.path.join(ref_root, "test", "mesh")):
            make_reference_meshes(work, ref_root)
            make_reference_partitions(ref_root)
    finally:
        shutil.rmtree(work, ignore_errors=True)


if __name__ == "__main__":
    main()
