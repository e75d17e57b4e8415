"""e3d_solver_run_noalloc against e3d_solver_run.

The allocation-free entry point serves callers that may not allocate device memory once their
set-up is done (a serving loop held to a fixed, pre-reserved memory budget, or code running where
the CUDA allocator may not be called).  It must give exactly what e3d_solver_run gives: it runs the
same kernels in the same order, only with its scratch (RMS partial sums and history) in a fixed
device array.  Checked on two calls in a row, so that the second call starts from a state and a
scratch array the first one left behind.  This file is collected last on purpose.
"""
import numpy as np
import pytest

from cases import CASES, STATE_KEYS, prepared
from euler3d_b200 import _lib
from euler3d_b200.solver import EulerSolver

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [_lib.PREC_FP64_EXACT, _lib.PREC_FP64, _lib.PREC_FP32_FLUX])
@pytest.mark.parametrize("name", ["channel", "tets"])
def test_noalloc_run_matches_run(name, precision):
    flow = CASES[name].flow(precision=precision, ordering=_lib.ORDER_SPATIAL)
    arrays = prepared(name)
    ref = EulerSolver(arrays, flow)
    new = EulerSolver(arrays, flow)
    for max_iter, sampling in ((6, 2), (5, 3)):  # two calls in a row
        st_ref = ref.run(max_iter, sampling=sampling)
        hist_ref = ref.rms_history()
        st_new, hist_new = new.run_noalloc(max_iter, sampling=sampling)
        # same kernels, same summation order: the results are identical (the tolerance of the
        # exact-mode tests, which is zero, holds for both precisions here)
        assert st_new["iterations"] == st_ref["iterations"] == max_iter
        assert np.array_equal(hist_new, hist_ref)
        assert (st_new["cl"], st_new["cd"], st_new["cm"]) == (st_ref["cl"], st_ref["cd"], st_ref["cm"])
        a, b = ref.get_state(), new.get_state()
        for k in STATE_KEYS:
            assert np.array_equal(a[k], b[k]), k
        # the wall Cp of the last sample is this call's (cleared at its start, as a run clears it)
        assert np.array_equal(new.wall_cp(), ref.wall_cp())


def test_noalloc_with_colouring():
    """A handle whose stage kernel is the face-colouring variant (chosen by an earlier run) runs it
    allocation-free too: its classes and accumulator were built when the variant was chosen."""
    name = "tets"
    flow = CASES[name].flow(precision=_lib.PREC_FP64, ordering=_lib.ORDER_SPATIAL)
    ref = EulerSolver(prepared(name), flow)
    new = EulerSolver(prepared(name), flow)
    ref.run(0, stage_kernel=_lib.KERNEL_COLOUR)
    new.run(0, stage_kernel=_lib.KERNEL_COLOUR)
    st_ref = ref.run(7)
    st_new, hist_new = new.run_noalloc(7)
    assert st_new["iterations"] == st_ref["iterations"] == 7
    assert np.array_equal(hist_new, ref.rms_history())
    a, b = ref.get_state(), new.get_state()
    for k in STATE_KEYS:
        assert np.array_equal(a[k], b[k]), k


def test_noalloc_leaves_no_stale_records(tmp_path):
    """After an allocation-free run the handle holds no RMS history or coefficient samples of it, so
    the queries of them must not hand back an earlier e3d_solver_run's records as this run's."""
    name = "channel"
    s = EulerSolver(prepared(name), CASES[name].flow())
    s.run(12, sampling=3)
    assert s.rms_history().size == 12 and s.coefficient_history().shape[0] == 4
    st, hist = s.run_noalloc(5, sampling=1)
    assert hist.size == 5 and st["iterations"] == 5
    assert s.rms_history().size == 0
    assert s.coefficient_history().shape[0] == 0
    with pytest.raises(_lib.E3DError) as e:
        s.write_outputs(str(tmp_path))
    assert e.value.status == _lib.E3D_ERR_INVALID_ARG
    s.run(4)  # a normal run records again
    assert s.rms_history().size == 4


def test_noalloc_rejects_beyond_limit():
    name = "channel"
    s = EulerSolver(prepared(name), CASES[name].flow())
    with pytest.raises(_lib.E3DError) as e:
        s.run_noalloc(65537)
    assert e.value.status == _lib.E3D_ERR_INVALID_ARG
    assert "limit" in str(e.value)
    st, hist = s.run_noalloc(3)  # the handle is still usable
    assert st["iterations"] == 3 and hist.size == 3
