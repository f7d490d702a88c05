"""The oracle's shared building blocks against independent closed forms.

The reference ships no golden vectors for this path, so these known-answer
checks pin the pieces of the CPU restatement that have an independent
definition: associated Legendre functions (scipy), the pivoted complex LU
solve (numpy/LAPACK), the three-node quadratic interpolation (exact on
quadratics) and complex division."""
import ctypes as C

import numpy as np
import pytest
from scipy.special import lpmv

from oracle import oracle as orc

dp = C.POINTER(C.c_double)


@pytest.fixture(scope="module")
def L():
    lib = orc.lib()
    lib.oracle_kat_plm.argtypes = [C.c_int, C.c_int, C.c_double, dp]
    lib.oracle_kat_glu.argtypes = [dp, dp, C.c_int]
    lib.oracle_kat_interp.argtypes = [C.c_double, dp, dp, C.c_int]
    lib.oracle_kat_interp.restype = C.c_double
    lib.oracle_kat_cdiv.argtypes = [dp, dp, dp]
    return lib


@pytest.mark.parametrize("m", [0, 1, 2, 3])
@pytest.mark.parametrize("x", [0.999, 0.7, 0.0, -0.3, -0.95])
def test_legendre_recurrence(L, m, x):
    lmax = 120
    out = np.zeros(lmax - m + 1)
    L.oracle_kat_plm(lmax, m, x, out.ctypes.data_as(dp))
    ref = np.array([lpmv(m, l, x) for l in range(m, lmax + 1)])
    scale = np.maximum(np.abs(ref), 1e-300)
    err = np.abs(out - ref) / np.maximum(scale, np.abs(ref).max() * 1e-12)
    assert err.max() < 1e-9, err.max()


@pytest.mark.parametrize("n", [3, 4])
def test_pivoted_lu_solve(L, n):
    rng = np.random.default_rng(n)
    for _ in range(20):
        A = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
        b = rng.normal(size=n) + 1j * rng.normal(size=n)
        a_f = np.ascontiguousarray(A.T.reshape(-1))  # column-major
        ai = np.empty(2 * n * n)
        ai[0::2], ai[1::2] = a_f.real, a_f.imag
        bi = np.empty(2 * n)
        bi[0::2], bi[1::2] = b.real, b.imag
        assert L.oracle_kat_glu(ai.ctypes.data_as(dp), bi.ctypes.data_as(dp), n) == 0
        x = bi[0::2] + 1j * bi[1::2]
        ref = np.linalg.solve(A, b)
        assert np.abs(x - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max())


def test_quadratic_interpolation_exact(L):
    rng = np.random.default_rng(7)
    for _ in range(50):
        c = rng.normal(size=3)
        rr = np.sort(rng.uniform(3000, 6000, size=3))
        r = rng.uniform(rr[0], rr[2])
        g = c[0] + c[1] * (rr - 4500) + c[2] * (rr - 4500) ** 2
        v = L.oracle_kat_interp(r, rr.ctypes.data_as(dp), g.ctypes.data_as(dp), 0)
        dv = L.oracle_kat_interp(r, rr.ctypes.data_as(dp), g.ctypes.data_as(dp), 1)
        assert v == pytest.approx(c[0] + c[1] * (r - 4500) + c[2] * (r - 4500) ** 2, rel=1e-9, abs=1e-9)
        assert dv == pytest.approx(c[1] + 2 * c[2] * (r - 4500), rel=1e-7, abs=1e-9)


def test_complex_division(L):
    rng = np.random.default_rng(3)
    q = np.zeros(2)
    for _ in range(200):
        a = rng.normal(size=2) * 10 ** rng.uniform(-5, 5)
        b = rng.normal(size=2) * 10 ** rng.uniform(-5, 5)
        L.oracle_kat_cdiv(a.ctypes.data_as(dp), b.ctypes.data_as(dp), q.ctypes.data_as(dp))
        ref = complex(*a) / complex(*b)
        assert abs(complex(*q) - ref) <= 4e-16 * abs(ref)
