"""A case given as partition files runs on one GPU: the merged mesh is an ordinary mesh to the solver,
bit for bit the oracle's result on the same arrays in FP64_EXACT."""
import numpy as np
import pytest

import pyoracle as po
from cases import STATE_KEYS
from euler3d_b200 import _lib
from euler3d_b200 import meshgen as mg
from euler3d_b200.solver import EulerSolver, FlowConfig, Mesh
from test_gpu_parity import RMS_RTOL, assert_state_equal, rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("family,parts", [("channel", 3), ("ogrid", 4)])
def test_partitioned_case_matches_oracle(family, parts, tmp_path):
    raw = mg.bump_channel(16, 8, 2) if family == "channel" else mg.biconvex_ogrid(24, 12, 2)
    paths = mg.write_partitions(raw, parts, str(tmp_path / "p#.par"))
    arrays = Mesh.read_partitions(paths).arrays()
    flow = FlowConfig(mach=0.7, aoa=1.5, cfl=1.2, precision=_lib.PREC_FP64_EXACT, ordering=_lib.ORDER_SPATIAL)
    m = po.Mesh(arrays)
    fl = po.flow(flow.mach, flow.aoa, flow.gamma, flow.cfl, flow.sref, flow.cref, flow.ref_point, tuple(flow.cl),
                 tuple(flow.cd), tuple(flow.cm))
    o = po.freestream(m, fl)
    _, ohist = po.run(m, fl, o, 25)
    s = EulerSolver(arrays, flow)
    assert s.run(25)["iterations"] == 25
    assert_state_equal(s.get_state(), o.a, m.n_cells, ghost_E_rtol=1e-13)
    assert rel_err(s.rms_history(), ohist) <= RMS_RTOL
