"""The reference's output files, host side: <partition>.bry from a prepared mesh equals the file
the reference's WriteSolution wrote (tests/golden/outputs/, made by tests/golden/make_golden.py)."""
import os

import pytest

from cases import CASES
from euler3d_b200.solver import Mesh

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "outputs")


@pytest.mark.parametrize("run", ["rk5_max_iter", "euler_residual_exit"])
def test_boundary_file_matches_reference(run, tmp_path):
    m = Mesh.from_raw(CASES["channel"].raw())
    p = tmp_path / "mesh.par.bry"
    m.write_boundary(str(p))
    assert p.read_bytes() == open(os.path.join(OUT, run, "mesh.par.bry"), "rb").read()


def test_boundary_file_bad_path():
    from euler3d_b200._lib import E3DError

    m = Mesh.from_raw(CASES["channel"].raw())
    with pytest.raises(E3DError):
        m.write_boundary("/nonexistent-dir/x.bry")
