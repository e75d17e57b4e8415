"""The drop-in, end to end: the reference's own solver program with EulerSolverGPU in place of
EulerSolver (oracle/_ref/e3d_gpu_main: euler3d_b200/adapter/gpu_main.cpp linked with the reference's
front end, built by `make -C oracle adapter`) writes, in FP64_EXACT, byte for byte the files the
reference program writes on the same case (oracle/_ref/e3d_ref_driver outputs): residuals.dat,
cp_part_0.dat, summary.txt (timings fixed), the .sol solution and the .bry boundary file."""
import os
import subprocess

import pytest

import pyoracle as po
from cases import CASES
from euler3d_b200 import meshgen as mg

GPU_MAIN = os.path.join(os.path.dirname(po.REF_DRIVER), "e3d_gpu_main")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (po.ref_available() and os.path.exists(GPU_MAIN)),
                                 reason="reference program or drop-in driver not built (make -C oracle ref adapter)")]

RUNS = {"rk5": dict(time_integration=2, max_iter=30, sampling=4),
        "euler_smooth": dict(time_integration=0, residual_smoothing=1, max_iter=40, sampling=5)}
FILES = ("output/residuals.dat", "output/cp_part_0.dat", "output/summary.txt", "mesh.par.sol", "mesh.par.bry")


@pytest.mark.parametrize("name", ["channel", "ogrid"])
@pytest.mark.parametrize("run", list(RUNS))
def test_dropin_program_matches_reference(name, run, tmp_path):
    case = CASES[name]
    raw = case.raw()
    cfg = mg.CaseConfig(mach=case.mach, aoa=case.aoa, cfl=case.cfl, orientation_cl=2, orientation_cd=0, **RUNS[run])
    dirs = {}
    for who in ("reference", "gpu"):
        d = tmp_path / who
        path = mg.write_case(raw, cfg, str(d))
        if who == "reference":
            po.ref_call("outputs", path, str(d / "dump"), "1234", "5678")
        else:
            subprocess.run([GPU_MAIN, path, "exact", "1234", "5678"], check=True, capture_output=True, text=True,
                           cwd=str(d), timeout=600)
        dirs[who] = d
    for f in FILES:
        assert (dirs["gpu"] / f).read_bytes() == (dirs["reference"] / f).read_bytes(), f
