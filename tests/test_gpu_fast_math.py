"""Accuracy of the FP64 mode's fast reciprocal and reciprocal square root.

The FP64 stage kernels take 1/x and 1/sqrt(x) from the single-precision hardware approximations
refined by one step of the truncated series of the exact correction (stage.cuh, rcp_nr and
rsqrt_nr).  ``e3d_fast_reciprocals`` evaluates them on the GPU beside CUDA's own double-precision
``1.0 / x`` and ``rsqrt(x)``; this test holds them to

* within 1 unit in the last place of the correctly rounded 1/x (numpy's IEEE division, which
  CUDA's ``1.0 / x`` must equal) and within 2 of 1/sqrt(x) (in extended precision) on arguments
  spread log-uniformly over 1e-29..1e29;
* CUDA's own results, bit for bit, wherever the seed is not used: zero, negative arguments of the
  square root, magnitudes outside [2^-99, 2^99), subnormals, Inf and NaN.
"""
import ctypes as C

import numpy as np
import pytest

from euler3d_b200 import _lib

pytestmark = pytest.mark.gpu


def evaluate(x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.empty(4 * x.size)
    lib = _lib.load()
    dp = C.POINTER(C.c_double)
    _lib.check(lib.e3d_fast_reciprocals(0, x.ctypes.data_as(dp), x.size, out.ctypes.data_as(dp)))
    out = out.reshape(-1, 4)
    return out[:, 0], out[:, 1], out[:, 2], out[:, 3]


def ulps(a, ref):
    return np.abs(a - ref) / np.spacing(np.abs(ref))


def test_in_range_accuracy():
    rng = np.random.default_rng(7)
    x = np.exp(rng.uniform(np.log(1e-29), np.log(1e29), 1_000_000))
    x = np.concatenate([x, -x[:1000], [1.0, 2.0, 0.5, 3.0, 1.4, 2.0 ** -98, 2.0 ** 98]])
    rcp, rcp_cuda, rsq, rsq_cuda = evaluate(x)
    assert np.array_equal(rcp_cuda, 1.0 / x)  # CUDA's IEEE division, correctly rounded
    assert ulps(rcp, 1.0 / x).max() <= 1.0
    pos = x > 0
    xl = x[pos].astype(np.longdouble)
    ref = (1 / np.sqrt(xl)).astype(np.float64)
    assert ulps(rsq[pos], ref).max() <= 2.0
    assert ulps(rsq_cuda[pos], ref).max() <= 2.0


def test_outside_the_seed_range_equals_cuda():
    tiny, huge = 2.0 ** -99, 2.0 ** 99
    x = np.array([0.0, -0.0, -1.0, -2.5e10, 5e-324, 1e-310, 1e-300, 1e-31, tiny * 0.75, huge, huge * 3,
                  1e30, 1e300, np.inf, -np.inf, np.nan])
    rcp, rcp_cuda, rsq, rsq_cuda = evaluate(x)
    assert np.array_equal(rcp, rcp_cuda, equal_nan=True)
    fallback = ~((x > 0) & (x >= tiny) & (x < huge))
    assert np.array_equal(rsq[fallback], rsq_cuda[fallback], equal_nan=True)
    # the reciprocal takes the seed for negative arguments too
    neg = np.array([-1.5, -3e-20, -7e20])
    rcp, rcp_cuda, _, _ = evaluate(neg)
    assert np.array_equal(rcp_cuda, 1.0 / neg) and ulps(rcp, 1.0 / neg).max() <= 1.0
