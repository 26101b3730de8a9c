"""The exponential of the exponential-sum family (gsb_exp.h: Tang's table-driven method,
compiled for the device and, identically, for the host): its error against long double over
1e8 arguments, and its special values."""

import ctypes
import math

import numpy as np


def _lib(oracle):
    L = oracle.lib()
    L.oracle_exp_check.argtypes = [ctypes.c_int64, ctypes.c_uint64, ctypes.c_double,
                                   ctypes.c_double, ctypes.POINTER(ctypes.c_double),
                                   ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int64)]
    L.oracle_exp_check.restype = ctypes.c_int
    L.oracle_exp.argtypes = [ctypes.c_double]
    L.oracle_exp.restype = ctypes.c_double
    return L


def test_exp_error_below_one_ulp(oracle):
    """At most 0.52 ulp on 1e8 arguments over the whole range of normal results (CUDA's own
    double exp is documented within 1 ulp); correctly rounded on all but a small fraction."""
    L = _lib(oracle)
    mu, wx, nn = ctypes.c_double(), ctypes.c_double(), ctypes.c_int64()
    n = 100_000_000
    assert L.oracle_exp_check(n, 20261204, -708.3, 709.7, ctypes.byref(mu), ctypes.byref(wx),
                              ctypes.byref(nn)) == 0
    assert mu.value <= 0.52, (mu.value, wx.value)
    assert nn.value <= n // 500, nn.value


def test_exp_special_values(oracle):
    e = _lib(oracle).oracle_exp
    assert e(0.0) == 1.0 and e(-0.0) == 1.0
    assert math.isnan(e(float("nan")))
    assert e(float("inf")) == float("inf") and e(-float("inf")) == 0.0
    assert e(710.0) == float("inf") and e(-746.0) == 0.0
    assert abs(e(709.78) / math.exp(709.78) - 1) < 3e-16
    # subnormal results: the one rounding of the final scaling
    for x in (-708.5, -720.0, -740.0, -744.4, -745.0):
        assert abs(e(x) - math.exp(x)) <= 2 ** -1074, x
    for x in (1e-300, -1e-300, 2.0 ** -54, 1.0, -1.0, 0.5, 10.0, -10.0):
        assert abs(e(x) / math.exp(x) - 1.0) <= 2.3e-16, x
    # monotone across the table's boundaries
    xs = np.linspace(-3.0, 3.0, 20001)
    ys = np.array([e(float(x)) for x in xs])
    assert np.all(np.diff(ys) > 0)
