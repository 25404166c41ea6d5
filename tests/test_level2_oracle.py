"""The oracle's Level-2 restatement (level2::gemv / ger, complex2::gemv /
geru / gerc) pinned on the reference's own tests (src/level2.rs:106-190,
src/complex2.rs:145-186), plus strided vectors and both layouts against a
float64 numpy evaluation. CPU only.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle


def test_gemv_notrans_colmajor_row_sums():  # src/level2.rs:110-131
    a = np.array([1.0, 4.0, 2.0, 5.0, 3.0, 6.0])
    x = np.ones(3)
    y = np.zeros(2)
    oracle.gemv(1, 0, 2, 3, 1.0, a, 2, x, 1, 0.0, y, 1)
    assert list(y) == [6.0, 15.0]


def test_gemv_trans_colmajor_column_sums():  # src/level2.rs:133-153
    a = np.array([1.0, 4.0, 2.0, 5.0, 3.0, 6.0])
    x = np.ones(2)
    y = np.zeros(3)
    oracle.gemv(1, 1, 2, 3, 1.0, a, 2, x, 1, 0.0, y, 1)
    assert list(y) == [5.0, 7.0, 9.0]


def test_gemv_rowmajor():  # src/level2.rs:155-176
    a = np.array([1.0, 2.0, 3.0, 4.0, 5.0, 6.0])
    x = np.array([1.0, 0.0, 1.0])
    y = np.zeros(2)
    oracle.gemv(0, 0, 2, 3, 1.0, a, 3, x, 1, 0.0, y, 1)
    assert list(y) == [4.0, 10.0]


def test_ger_basic():  # src/level2.rs:178-188
    x = np.array([1.0, 2.0])
    y = np.array([3.0, 4.0])
    a = np.zeros(4)
    oracle.ger(1, 2, 2, 1.0, x, 1, y, 1, a, 2)
    assert list(a) == [3.0, 6.0, 4.0, 8.0]


def test_complex_gemv_notrans():  # src/complex2.rs:150-172
    a = np.array([1 + 0j, 0 + 1j])
    x = np.array([1 + 0j, 1 + 0j])
    y = np.zeros(1, dtype=np.complex128)
    oracle.gemv(1, 0, 1, 2, 1 + 0j, a, 1, x, 1, 0j, y, 1)
    assert y[0] == 1 + 1j


def test_gerc_conjugates_y():  # src/complex2.rs:174-183
    x = np.array([1 + 0j])
    y = np.array([0 + 1j])
    a = np.zeros(1, dtype=np.complex128)
    oracle.ger(1, 1, 1, 1 + 0j, x, 1, y, 1, a, 1, conj=True)
    assert a[0] == -1j


def _dense(layout, m, n, a, lda):
    if layout == 1:
        return np.array([[a[i + j * lda] for j in range(n)] for i in range(m)])
    return np.array([[a[i * lda + j] for j in range(n)] for i in range(m)])


@pytest.mark.parametrize("dtype", [np.float64, np.complex128])
@pytest.mark.parametrize("layout", [0, 1])
@pytest.mark.parametrize("trans", [0, 1, 2])
def test_gemv_strided_against_numpy(dtype, layout, trans):
    cx = np.issubdtype(dtype, np.complexfloating)
    if trans == 2 and not cx:
        pytest.skip("ConjTrans == Trans for real types")
    rng = np.random.default_rng(7 + layout + 2 * trans)
    m, n, incx, incy = 37, 29, 2, 3
    lda = (n if layout == 0 else m) + 4
    a = rng.standard_normal(lda * (n if layout == 1 else m)) + (1j * rng.standard_normal(lda * (n if layout == 1 else m)) if cx else 0)
    a = a.astype(dtype)
    lenx, leny = (m, n) if trans else (n, m)
    x = (rng.standard_normal(lenx * incx) + (1j * rng.standard_normal(lenx * incx) if cx else 0)).astype(dtype)
    y0 = (rng.standard_normal(leny * incy) + (1j * rng.standard_normal(leny * incy) if cx else 0)).astype(dtype)
    alpha, beta = (1.5 - 0.5j, -0.25 + 1j) if cx else (1.5, -0.25)
    y = y0.copy()
    oracle.gemv(layout, trans, m, n, alpha, a, lda, x, incx, beta, y, incy)
    A = _dense(layout, m, n, a, lda)
    op = A.conj().T if trans == 2 else (A.T if trans == 1 else A)
    ref = alpha * (op @ x[::incx][:lenx]) + beta * y0[::incy][:leny]
    assert np.allclose(y[::incy][:leny], ref, rtol=1e-12, atol=1e-12)
    untouched = np.ones(len(y), dtype=bool)
    untouched[::incy] = False
    assert np.array_equal(y[untouched], y0[untouched])


def test_ger_exact_fma_rounding():
    """a_ij = fma(alpha * x_i, y_j, a_ij): alpha*x_i rounded once, then one fused step."""
    rng = np.random.default_rng(3)
    m, n = 9, 7
    x, y = rng.standard_normal(m), rng.standard_normal(n)
    a0 = rng.standard_normal(m * n)
    a = a0.copy()
    oracle.ger(1, m, n, 0.7, x, 1, y, 1, a, m)
    from fractions import Fraction

    def fma(p, q, r):  # exact product and sum, one rounding
        return float(Fraction(float(p)) * Fraction(float(q)) + Fraction(float(r)))

    for i in range(m):
        axi = 0.7 * x[i]
        for j in range(n):
            assert a[i + j * m] == fma(axi, y[j], a0[i + j * m])
