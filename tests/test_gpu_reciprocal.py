"""The reciprocal and square root the stage kernels use in their flux and
wave-speed formulas (frcp and fsqrt in frforge_b200/csrc/frg_device.cuh:
hardware estimates refined by Newton-Raphson and Goldschmidt iterations)
against CUDA's correctly rounded division and sqrt on the same device:
within 1 ulp over the operand ranges the kernels use, and non-finite where
the exact result is."""
import ctypes as C

import numpy as np
import pytest

from frforge_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _check(x, name="frg_internal_reciprocal_check"):
    lib = L.load()
    fn = getattr(lib, name)
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(C.c_double)] * 3 + [C.c_size_t]
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.empty_like(x)
    q = np.empty_like(x)
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
    assert fn(dp(x), dp(y), dp(q), x.size) == 0
    return y, q


def _ulps(a, b):
    ia = a.view(np.int64)
    ib = b.view(np.int64)
    return np.abs(ia - ib)


def test_reciprocal_within_one_ulp():
    rng = np.random.default_rng(20261203)
    # random mantissas over the exponent range the kernels meet, both signs,
    # plus the floors and guards of the flux formulas
    e = rng.integers(-1000, 1000, size=200000)
    m = rng.uniform(1.0, 2.0, size=e.size)
    x = np.ldexp(m, e) * np.where(rng.random(e.size) < 0.5, -1.0, 1.0)
    x = np.concatenate([x, [2.220446049250313e-16, 1.0, -1.0, 0.125, 3.0, 1e-300, 1e300, 1.4, 0.4]])
    y, q = _check(x)
    assert np.all(np.isfinite(y)) and np.all(np.isfinite(q))
    assert int(_ulps(y, q).max()) <= 1
    # most results are the correctly rounded quotient itself
    assert np.mean(y == q) > 0.9


def test_reciprocal_non_finite_cases():
    y, q = _check(np.array([0.0, np.inf, -np.inf, np.nan]))
    # the exact division gives +inf, 0, -0, NaN; frcp gives non-finite or
    # NaN there, which the stage kernels flag like the exact infinities
    assert np.isnan(y[0]) and np.isinf(q[0])
    assert np.isnan(y[3]) and np.isnan(q[3])


def test_sqrt_within_one_ulp():
    rng = np.random.default_rng(20261204)
    e = rng.integers(-1000, 1000, size=200000)
    x = np.ldexp(rng.uniform(1.0, 2.0, size=e.size), e)
    # sound-speed operands gamma p / rho with floored p and rho
    x = np.concatenate([x, [1.4 * 2.220446049250313e-16, 1.4, 0.56, 1.4e-16 / 3.0, 4.0, 2.0, 1e-300, 1e300]])
    y, q = _check(x, "frg_internal_sqrt_check")
    assert np.all(np.isfinite(y)) and np.all(np.isfinite(q))
    assert int(_ulps(y, q).max()) <= 1
    assert np.mean(y == q) > 0.9
    y, q = _check(np.array([np.nan, np.inf]), "frg_internal_sqrt_check")
    assert np.isnan(y[0]) and not np.isfinite(y[1])
