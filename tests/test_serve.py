"""Request streams and request meshes of the serving loop (host side)."""
import math

import numpy as np
import pytest

from euler3d_b200 import _lib, serve


def test_stream_is_seeded_and_in_range():
    a = serve.request_stream(200, rate=20.0, cells=(10_000, 2_000_000), seed=4)
    b = serve.request_stream(200, rate=20.0, cells=(10_000, 2_000_000), seed=4)
    assert a == b
    arr = np.array([r.arrival for r in a])
    assert arr[0] == 0.0 and np.all(np.diff(arr) >= 0)
    # Poisson arrivals: mean gap 1 / rate
    assert abs(np.mean(np.diff(arr)) - 1 / 20.0) < 0.2 / 20.0
    cells = np.array([r.cells for r in a])
    assert cells.min() >= 10_000 and cells.max() <= 2_000_000
    # log-uniform: the median is near the geometric mean of the bounds
    assert abs(math.log(np.median(cells)) - 0.5 * math.log(10_000 * 2_000_000)) < 0.6
    assert {r.drop for r in a} == {1e-6, 1e-8}
    assert all(0.3 <= r.mach <= 0.85 and -4 <= r.aoa <= 6 for r in a)
    assert {r.family for r in a} == {"channel", "ogrid"}


def test_burst_stream():
    a = serve.request_stream(5, rate=0.0, seed=1)
    assert all(r.arrival == 0.0 for r in a)


@pytest.mark.parametrize("family", ["channel", "ogrid"])
@pytest.mark.parametrize("cells", [900, 5000, 40000])
def test_request_mesh_size(family, cells):
    req = serve.SolveRequest(0, 0.0, family, cells, 0.5, 0.0, 1e-6, seed=3)
    a = serve._prepare(req)
    assert abs(a["n_cells"] - cells) <= 0.15 * cells
    assert np.all(a["cell_volume"] > 0)


def test_summarize():
    rs = [serve.SolveResult(i, 100, float(i), float(i), float(i) + 1 + i, 10, 1, 0, 0, 0, 0, 0, 0)
          for i in range(4)]
    s = serve.summarize(rs)
    assert s["solves"] == 4 and s["seconds"] == 7.0
    assert s["p50_latency_s"] == 2.5 and abs(s["solves_per_s"] - 4 / 7) < 1e-12
    assert s["cell_iterations"] == 4000
    assert (s["converged"], s["capped"], s["diverged"]) == (4, 0, 0)


def test_footprint_estimate_grows_with_size():
    e1 = serve.footprint_estimate(1000, 3000, _lib.PREC_FP64)
    e2 = serve.footprint_estimate(2000, 6000, _lib.PREC_FP64)
    e3 = serve.footprint_estimate(2000, 6000, _lib.PREC_FP32_FLUX)
    assert e1 < e2 < e3
