"""The pivot reciprocal of the diagonal-block kernels (GPU).

The elimination step of the diagonal-block kernels forms 1/d with the
hardware reciprocal approximation refined by two Newton-Raphson steps
instead of the IEEE division.  It must stay within one ulp of the IEEE
quotient 1.0 / d computed on the device, over pivots of every magnitude and
sign, and equal it exactly where it falls back to the quotient (zero,
subnormal, huge, infinite and NaN values).
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _check(x):
    import sam_lib_b200 as spr
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.zeros(2 * x.size)
    lib = spr.load(8)
    lib.spr_b200_recip_check.argtypes = [C.c_void_p, C.c_int64, C.c_void_p]
    assert lib.spr_b200_recip_check(x.ctypes.data, x.size, out.ctypes.data) == 0
    return out[0::2], out[1::2]


def test_reciprocal_within_one_ulp():
    rng = np.random.default_rng(11)
    mag = 10.0 ** rng.uniform(-300, 300, size=200000)
    x = np.concatenate([mag, -mag, 1.0 + rng.uniform(-1e-3, 1e-3, 50000), np.arange(1, 5000, dtype=float)])
    r, q = _check(x)
    assert np.all(np.isfinite(r))
    ulps = np.abs(r - q) / np.spacing(np.abs(q))
    assert ulps.max() <= 1.0, ulps.max()
    # almost always the correctly rounded quotient itself
    assert np.mean(r == q) > 0.99


def test_reciprocal_special_values_take_the_quotient():
    x = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 5e-324, 1e-310, -1e-310, 1.5e308, -1.7e308])
    r, q = _check(x)
    same = (r == q) | (np.isnan(r) & np.isnan(q))
    assert np.all(same), (r, q)
    assert np.array_equal(np.signbit(r[:4]), np.signbit(q[:4]))
