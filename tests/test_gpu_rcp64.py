"""The FP64 link reciprocal of the tolerance solve against IEEE division.

The FP64 outer residual evaluates each harmonic-mean link weight k_i k_j /
(k_i + k_j) with a hardware reciprocal refined by two Newton steps instead of
an IEEE division.  This test evaluates both on the device over the range of
kappa sums the solve produces (kappa normalised to mean 1: sums of two
voxels' kappa in [0.3, 6] on the three-material mix) and over every binade
of the double range, and bounds the difference at 1 ulp of the IEEE
quotient; subnormal and huge inputs, which the hardware approximation
flushes, must equal the IEEE quotient exactly.
"""
import numpy as np
import pytest

from pfsf_b200 import capi

pytestmark = pytest.mark.gpu


def _eval(s):
    L = capi.load()
    s = np.ascontiguousarray(s, np.float64)
    a = np.zeros_like(s)
    b = np.zeros_like(s)
    rc = L.pfsf_debug_rcp64(s.ctypes.data, a.ctypes.data, b.ctypes.data, s.size)
    assert rc == capi.PFSF_OK
    return a, b


def _ulps(a, b):
    ia = a.view(np.int64)
    ib = b.view(np.int64)
    return np.abs(ia - ib)


def test_rcp64_within_one_ulp_of_ieee(lib_built):
    rng = np.random.default_rng(5)
    kappa_sums = rng.uniform(0.3, 6.0, 1 << 20)
    wide = np.exp(rng.uniform(np.log(2.0 ** -1021), np.log(2.0 ** 1019), 1 << 20))
    binades = np.ldexp(1.0, np.arange(-1022, 1021)) * rng.uniform(1.0, 2.0, 2043)
    s = np.concatenate([kappa_sums, wide, binades, [1.0, 2.0, 0.5, 3.0, 1.0 / 3.0]])
    a, b = _eval(s)
    assert np.all(np.isfinite(a))
    u = _ulps(a, b)
    assert u.max() <= 1, f"max ulp difference {u.max()} at s={s[np.argmax(u)]!r}"
    # on the solve's own range the refined reciprocal is almost always exact
    uk = u[: kappa_sums.size]
    assert np.mean(uk == 0) > 0.99


def test_rcp64_extremes_take_ieee_division(lib_built):
    tiny = np.array([5e-324, 1e-310, 2.2250738585072e-308, np.nextafter(2.0 ** -1022, 0.0)])
    huge = np.array([2.0 ** 1020 * 1.5, 1e308, np.finfo(np.float64).max])
    s = np.concatenate([tiny, huge])
    a, b = _eval(s)
    assert np.array_equal(a.view(np.int64), b.view(np.int64)), (a, b)
    assert np.all(np.isinf(a[:1]))  # 1 / 5e-324 overflows in IEEE too
    assert np.all(a[len(tiny):] > 0.0)
