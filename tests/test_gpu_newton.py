"""The contracted build's reciprocal and square root (rcp_newton and
sqrt_newton in common.cuh: the hardware estimate refined by Newton-Raphson
steps) against IEEE 1/x and sqrt(x) over the ranges the solvers meet (and
well beyond): within 2 ulp, with sqrt(0) = 0."""
import ctypes

import numpy as np
import pytest

from classic_b200 import _lib

pytestmark = pytest.mark.gpu


def _ulps(a, b):
    return np.abs(a - b) / np.spacing(np.abs(b))


def test_newton_reciprocal_and_root_within_two_ulp():
    rng = np.random.default_rng(3)
    x = np.concatenate([10.0 ** rng.uniform(-30, 30, 200000), rng.uniform(0.5, 2.0, 100000),
                        np.array([1.0, 2.0, 4.0, 0.25, 1.4, 0.4, 1e-300, 1e300])])
    rcp = np.empty_like(x)
    root = np.empty_like(x)
    P = ctypes.POINTER(ctypes.c_double)
    lib = _lib.load()
    assert lib.claw_check_newton(x.ctypes.data_as(P), x.size, rcp.ctypes.data_as(P),
                                 root.ctypes.data_as(P)) == 0
    ok = (x > 1e-290) & (x < 1e290)  # away from the ftz / overflow edges of the estimate
    ur, us = _ulps(rcp[ok], 1.0 / x[ok]), _ulps(root[ok], np.sqrt(x[ok]))
    print(f"max ulp error: reciprocal {ur.max():.2f}, square root {us.max():.2f}")
    assert ur.max() <= 2.0 and us.max() <= 2.0
    z = np.zeros(4)
    r0, s0 = np.empty(4), np.empty(4)
    assert lib.claw_check_newton(z.ctypes.data_as(P), 4, r0.ctypes.data_as(P), s0.ctypes.data_as(P)) == 0
    assert np.all(s0 == 0.0)
