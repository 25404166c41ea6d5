"""GPU tests of Level 2 (gemv, ger, geru, gerc) through the C ABI against
the oracle's restatement of rblas (src/level2.rs, src/complex2.rs).

Tolerances: a gemv output is a length-K dot product (K = n for NoTrans, m
for Trans) summed in a different order than rblas's, so each element must
lie within 4*K*u * (|alpha| * sum_k |a_k||x_k| + |beta| |y0|) of the
oracle's (u of the dtype). The rank-1 updates compute every element as
rblas does, so they must match the oracle bit for bit. Also: the
reference's own known answers, strided vectors with untouched gaps, both
layouts, beta/alpha special values (beta = 0 ignores NaN in y; complex
always runs the beta pass), and the argument checks.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from rblas_b200 import complex2, level2
from rblas_b200.error import BufferTooSmall, InvalidLeadingDim, ZeroStride

pytestmark = pytest.mark.gpu


def _u(dt):
    return 2.0 ** -24 if np.dtype(dt) in (np.float32, np.complex64) else 2.0 ** -53


def _rand(rng, n, dt):
    v = rng.standard_normal(n)
    if np.issubdtype(np.dtype(dt), np.complexfloating):
        v = v + 1j * rng.standard_normal(n)
    return v.astype(dt)


def _dense(layout, m, n, a, lda):
    idx = (np.arange(m)[:, None] + np.arange(n)[None, :] * lda) if layout == 1 else \
        (np.arange(m)[:, None] * lda + np.arange(n)[None, :])
    return a[idx]


def _mod(dt):
    return complex2 if np.issubdtype(np.dtype(dt), np.complexfloating) else level2


@pytest.mark.parametrize("dt", [np.float32, np.float64, np.complex64, np.complex128])
@pytest.mark.parametrize("layout", [0, 1])
@pytest.mark.parametrize("trans", [0, 1, 2])
@pytest.mark.parametrize("shape", [(1, 1), (37, 29), (300, 5), (5, 300), (1000, 777)])
def test_gemv_matches_oracle(dt, layout, trans, shape):
    cx = np.issubdtype(np.dtype(dt), np.complexfloating)
    if trans == 2 and not cx:
        pytest.skip("ConjTrans == Trans for real types")
    m, n = shape
    rng = np.random.default_rng(11 + m + 3 * n + layout + 7 * trans)
    incx, incy = 2, 3
    lda = (n if layout == 0 else m) + 3
    a = _rand(rng, lda * (m if layout == 0 else n), dt)
    lenx, leny = (m, n) if trans else (n, m)
    x = _rand(rng, (lenx - 1) * incx + 1, dt)
    y0 = _rand(rng, (leny - 1) * incy + 1, dt)
    alpha, beta = ((1.25 - 0.5j, -0.75 + 0.25j) if cx else (1.25, -0.75))
    got, ref = y0.copy(), y0.copy()
    _mod(dt).gemv(layout, trans, m, n, alpha, a, lda, x, incx, beta, got, incy)
    oracle.gemv(layout, trans, m, n, alpha, a, lda, x, incx, beta, ref, incy)
    A = _dense(layout, m, n, a, lda)
    op = A.conj().T if trans == 2 else (A.T if trans else A)
    scale = abs(alpha) * (np.abs(op) @ np.abs(x[::incx][:lenx])) + abs(beta) * np.abs(y0[::incy][:leny])
    tol = 4 * max(lenx, 1) * _u(dt) * scale + 1e-300
    assert np.all(np.abs(got[::incy][:leny].astype(np.complex128) - ref[::incy][:leny]) <= tol)
    gaps = np.ones(len(y0), dtype=bool)
    gaps[::incy] = False
    assert np.array_equal(got[gaps], y0[gaps])


def test_gemv_notrans_colmajor_single_range_is_bit_exact():
    """One column range per row (few columns): the sum runs in rblas's order."""
    rng = np.random.default_rng(5)
    m, n = 200000, 8
    a, x, y0 = rng.standard_normal(m * n), rng.standard_normal(n), rng.standard_normal(m)
    got, ref = y0.copy(), y0.copy()
    level2.gemv(1, 0, m, n, 0.5, a, m, x, 1, 2.0, got, 1)
    oracle.gemv(1, 0, m, n, 0.5, a, m, x, 1, 2.0, ref, 1)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("dt", [np.float32, np.float64, np.complex64, np.complex128])
@pytest.mark.parametrize("layout", [0, 1])
@pytest.mark.parametrize("conj", [False, True])
def test_rank1_update_is_bit_exact(dt, layout, conj):
    cx = np.issubdtype(np.dtype(dt), np.complexfloating)
    if conj and not cx:
        pytest.skip("gerc is complex only")
    rng = np.random.default_rng(21 + layout + 2 * conj)
    for m, n in [(1, 1), (33, 17), (700, 300)]:
        incx, incy = 3, 2
        lda = (n if layout == 0 else m) + 5
        x = _rand(rng, (m - 1) * incx + 1, dt)
        y = _rand(rng, (n - 1) * incy + 1, dt)
        a0 = _rand(rng, lda * (m if layout == 0 else n), dt)
        alpha = 0.75 + 1.5j if cx else 0.75
        got, ref = a0.copy(), a0.copy()
        if cx:
            (complex2.gerc if conj else complex2.geru)(layout, m, n, alpha, x, incx, y, incy, got, lda)
        else:
            level2.ger(layout, m, n, alpha, x, incx, y, incy, got, lda)
        oracle.ger(layout, m, n, alpha, x, incx, y, incy, ref, lda, conj=conj)
        assert np.array_equal(got, ref), (m, n)


def test_reference_known_answers():
    # src/level2.rs:110-188, src/complex2.rs:150-183
    y = np.zeros(2)
    level2.gemv(1, 0, 2, 3, 1.0, np.array([1.0, 4.0, 2.0, 5.0, 3.0, 6.0]), 2, np.ones(3), 1, 0.0, y, 1)
    assert list(y) == [6.0, 15.0]
    y = np.zeros(3)
    level2.gemv(1, 1, 2, 3, 1.0, np.array([1.0, 4.0, 2.0, 5.0, 3.0, 6.0]), 2, np.ones(2), 1, 0.0, y, 1)
    assert list(y) == [5.0, 7.0, 9.0]
    y = np.zeros(2)
    level2.gemv(0, 0, 2, 3, 1.0, np.arange(1.0, 7.0), 3, np.array([1.0, 0.0, 1.0]), 1, 0.0, y, 1)
    assert list(y) == [4.0, 10.0]
    a = np.zeros(4)
    level2.ger(1, 2, 2, 1.0, np.array([1.0, 2.0]), 1, np.array([3.0, 4.0]), 1, a, 2)
    assert list(a) == [3.0, 6.0, 4.0, 8.0]
    y = np.zeros(1, dtype=np.complex128)
    complex2.gemv(1, 0, 1, 2, 1, np.array([1 + 0j, 1j]), 1, np.array([1 + 0j, 1 + 0j]), 1, 0, y, 1)
    assert y[0] == 1 + 1j
    a = np.zeros(1, dtype=np.complex128)
    complex2.gerc(1, 1, 1, 1, np.array([1 + 0j]), 1, np.array([1j]), 1, a, 1)
    assert a[0] == -1j


def test_special_alpha_beta_and_zero_stride_x():
    rng = np.random.default_rng(9)
    m, n = 64, 48
    a, x = rng.standard_normal(m * n), rng.standard_normal(n)
    y = np.full(m, np.nan)
    level2.gemv(1, 0, m, n, 1.0, a, m, x, 1, 0.0, y, 1)  # beta = 0: y never read
    assert not np.any(np.isnan(y))
    y0 = rng.standard_normal(m)
    y = y0.copy()
    level2.gemv(1, 0, m, n, 0.0, a, m, x, 1, 1.0, y, 1)  # alpha = 0, beta = 1: untouched
    assert np.array_equal(y, y0)
    got, ref = y0.copy(), y0.copy()
    level2.gemv(1, 0, m, n, 1.5, a, m, x[:1], 0, -1.0, got, 1)  # incx = 0: x[0] everywhere
    oracle.gemv(1, 0, m, n, 1.5, a, m, x[:1], 0, -1.0, ref, 1)
    assert np.allclose(got, ref, rtol=1e-13, atol=1e-13)
    # complex: the beta pass runs even for beta = 1, so an infinite entry
    # turns into NaN (0 * inf in the complex multiply) as in rblas
    yc = np.array([complex(np.inf, 1.0), 1 + 1j])
    ref = yc.copy()
    complex2.gemv(1, 0, 2, 1, 0, np.ones(2, dtype=np.complex128), 2, np.ones(1, dtype=np.complex128), 1, 1, yc, 1)
    oracle.gemv(1, 0, 2, 1, 0, np.ones(2, dtype=np.complex128), 2, np.ones(1, dtype=np.complex128), 1, 1, ref, 1)
    assert np.array_equal(yc, ref, equal_nan=True)


def test_argument_checks():
    a, x, y = np.zeros(12), np.zeros(4), np.zeros(3)
    with pytest.raises(InvalidLeadingDim):
        level2.gemv(1, 0, 3, 4, 1.0, a, 2, x, 1, 0.0, y, 1)
    with pytest.raises(BufferTooSmall):
        level2.gemv(1, 0, 3, 4, 1.0, a[:11], 3, x, 1, 0.0, y, 1)
    with pytest.raises(BufferTooSmall):
        level2.gemv(1, 0, 3, 4, 1.0, a, 3, x, 2, 0.0, y, 1)
    with pytest.raises(ZeroStride):
        level2.gemv(1, 0, 3, 4, 1.0, a, 3, x, 1, 0.0, y, 0)
    with pytest.raises(BufferTooSmall):
        level2.ger(1, 3, 4, 1.0, x[:3], 1, x[:3], 1, a, 3)
