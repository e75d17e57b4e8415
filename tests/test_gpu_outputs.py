"""The reference's output files written from the GPU solver (FP64_EXACT) are byte for byte the files
the reference's own writers produced for the same runs (tests/golden/outputs/, made by
tests/golden/make_golden.py from the reference solver): residuals.dat, cp_part_0.dat, summary.txt
and the .sol solution."""
import json
import os

import numpy as np
import pytest

from cases import CASES, prepared
from euler3d_b200 import _lib
from euler3d_b200.solver import EulerSolver, FlowConfig

pytestmark = pytest.mark.gpu

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "outputs")
FILES = ("residuals.dat", "cp_part_0.dat", "summary.txt", "mesh.par.sol")


def solve(run):
    cfg = json.load(open(os.path.join(OUT, run, "run.json")))
    case = CASES[cfg["case"]]
    cl, cd, cm = FlowConfig.orientation(2, 0)
    integ = _lib.INTEGRATOR_EULER if cfg["time_integration"] == 0 else _lib.INTEGRATOR_RK5
    flow = case.flow(precision=_lib.PREC_FP64_EXACT, integrator=integ, cl=cl, cd=cd, cm=cm,
                     ref_point=(0.25, 0.0, 0.0))
    s = EulerSolver(prepared(cfg["case"]), flow)
    st = s.run(cfg["max_iter"], sampling=cfg["sampling"], min_residual=cfg["min_residual"])
    return s, st, cfg


@pytest.mark.parametrize("run", ["rk5_max_iter", "euler_residual_exit"])
def test_output_files_match_reference(run, tmp_path):
    s, st, cfg = solve(run)
    s.write_outputs(str(tmp_path), partition_file=str(tmp_path / "mesh.par"), solver_ms=cfg["solver_ms"],
                    total_ms=cfg["total_ms"], n_cores=1)
    for f in FILES:
        got = (tmp_path / f).read_bytes()
        want = open(os.path.join(OUT, run, f), "rb").read()
        assert got == want, f"{run}/{f} differs"


def test_coefficient_history_and_cp():
    s, st, cfg = solve("rk5_max_iter")
    h = s.coefficient_history()
    assert h.shape == (cfg["max_iter"] // cfg["sampling"], 7)
    assert np.array_equal(h[:, 0], np.arange(1, h.shape[0] + 1) * cfg["sampling"])
    assert np.array_equal(h[-1, 1:4], np.array(st["force"]))
    cp = s.wall_cp()
    assert cp.size == prepared("channel")["wall_ghost"].size and np.all(np.isfinite(cp))
    # Cp of the last sample, not of the final state (the reference's PrintCp): rerun one more iteration
    s.run(1, sampling=1000)
    assert not s.wall_cp().any()  # a fresh run before its first sample: zeros


def test_write_errors():
    s, _, _ = solve("rk5_max_iter")
    with pytest.raises(_lib.E3DError):
        s.write_outputs("/nonexistent-dir")
