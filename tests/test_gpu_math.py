"""The library's own sin/cos/asin (range-reduced Taylor series used by the
throughput forms) against CUDA's functions, on the device (GPU).

Bounds: float results within 3e-7 absolute of sin/cos (2.5 ulp at 1) and
2.5e-7 relative for asin; double within 1e-15 absolute / 5e-16 relative.  The
mixed form's 1 - a0/|a| (Newton-refined hardware reciprocal square root and
reciprocal) within 5e-7 relative (about 8 ulp) of the same expression in double.
"""
import ctypes

import pytest

pytestmark = pytest.mark.gpu


def test_elementary_functions_against_cuda():
    from gftevolver_b200 import _lib
    lib = _lib.load()
    out = (ctypes.c_double * 9)()
    _lib.check(lib.gft_selftest_math(0, out))
    f_sin, f_cos, f_sin1, d_sin, d_cos, d_sin1, f_asin, d_asin, f_omc = list(out)
    assert f_sin <= 3e-7 and f_cos <= 3e-7 and f_sin1 <= 3e-7, (f_sin, f_cos, f_sin1)
    assert d_sin <= 1e-15 and d_cos <= 1e-15 and d_sin1 <= 1e-15, (d_sin, d_cos, d_sin1)
    assert f_asin <= 2.5e-7, f_asin
    assert d_asin <= 5e-16, d_asin
    assert 0.0 < f_omc <= 5e-7, f_omc
