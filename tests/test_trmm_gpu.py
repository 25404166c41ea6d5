"""GPU tests of trmm (B := alpha*op(A)*B or alpha*B*op(A), A triangular).
rblas has no trmm (its README lists it as remaining Level 3), so the oracle
is the textbook definition restated in oracle/ (real types) and a dense
numpy evaluation (complex). Tolerance: normwise 4*q*u relative to
|alpha| ||A|| ||B|| (q = order of A). Also: the unreferenced triangle and,
for Unit, the diagonal are never read (filled with NaN here); alpha = 0
gives zeros; argument checks."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from rblas_b200 import complex3, level3
from rblas_b200.error import InvalidLeadingDim

pytestmark = pytest.mark.gpu


def _u(dt):
    return 2.0 ** -24 if np.dtype(dt) in (np.float32, np.complex64) else 2.0 ** -53


def _tri(rng, q, lda, uplo, diag, dt, poison=True):
    cx = np.issubdtype(np.dtype(dt), np.complexfloating)
    a = rng.standard_normal((lda, q)) + (1j * rng.standard_normal((lda, q)) if cx else 0)
    mask = np.triu(np.ones((q, q), bool)) if uplo == 0 else np.tril(np.ones((q, q), bool))
    if diag == 1:
        mask &= ~np.eye(q, dtype=bool)
    if poison:
        a[:q][~mask] = np.nan  # never read
    return np.asfortranarray(a.astype(dt)).reshape(-1, order="F"), mask


def _dense_op(a, lda, q, mask, diag, trans):
    A = a.reshape(q, lda).T[:q, :q].copy()  # column-major view
    A = np.where(mask, A, 0)
    if diag == 1:
        A = A + np.eye(q)
    return A.conj().T if trans == 2 else (A.T if trans == 1 else A)


@pytest.mark.parametrize("dt", [np.float32, np.float64, np.complex64, np.complex128])
@pytest.mark.parametrize("side", [0, 1])
@pytest.mark.parametrize("uplo", [0, 1])
@pytest.mark.parametrize("trans", [0, 1, 2])
def test_trmm_parity(dt, side, uplo, trans):
    cx = np.issubdtype(np.dtype(dt), np.complexfloating)
    if trans == 2 and not cx:
        pytest.skip("ConjTrans == Trans for real types")
    rng = np.random.default_rng(100 + side + 2 * uplo + 4 * trans)
    for (m, n) in [(1, 1), (70, 33), (257, 130)]:
        for diag in (0, 1):
            q = m if side == 0 else n
            lda, ldb = q + 2, m + 3
            a, mask = _tri(rng, q, lda, uplo, diag, dt)
            b0 = (rng.standard_normal(ldb * n) + (1j * rng.standard_normal(ldb * n) if cx else 0)).astype(dt)
            alpha = (0.75 - 0.5j) if cx else 0.75
            b = b0.copy()
            (complex3 if cx else level3).trmm(side, uplo, trans, diag, m, n, alpha, a, lda, b, ldb)
            B0 = b0.reshape(n, ldb).T[:m, :]
            opA = _dense_op(a, lda, q, mask, diag, trans)
            ref = alpha * (opA @ B0 if side == 0 else B0 @ opA)
            if not cx:
                rb = b0.copy()
                oracle.trmm(side, uplo, trans, diag, m, n, alpha, np.nan_to_num(a), lda, rb, ldb)
                ref = rb.reshape(n, ldb).T[:m, :]
            got = b.reshape(n, ldb).T[:m, :]
            den = abs(alpha) * np.linalg.norm(opA) * np.linalg.norm(B0)
            assert np.linalg.norm(got.astype(np.complex128) - ref) <= 4 * q * _u(dt) * den + 1e-300, (m, n, diag)
            pad = b.reshape(n, ldb).T[m:, :]
            assert np.array_equal(pad, b0.reshape(n, ldb).T[m:, :])  # rows beyond m untouched


@pytest.mark.parametrize("dt", [np.float32, np.float64, np.complex128])
@pytest.mark.parametrize("side", [0, 1])
@pytest.mark.parametrize("uplo", [0, 1])
@pytest.mark.parametrize("trans", [0, 1, 2])
def test_trmm_recursive_parity(dt, side, uplo, trans):
    """Order 1100 (two 512-row leaves and a ragged 76-row one): the halves
    are multiplied by their diagonal blocks and the off-diagonal products
    added in the order that reads each half before it changes."""
    cx = np.issubdtype(np.dtype(dt), np.complexfloating)
    if trans == 2 and not cx:
        pytest.skip("ConjTrans == Trans for real types")
    rng = np.random.default_rng(200 + side + 2 * uplo + 4 * trans)
    q, nr = 1100, 40
    m, n = (q, nr) if side == 0 else (nr, q)
    for diag in (0, 1):
        lda, ldb = q + 2, m + 3
        a, mask = _tri(rng, q, lda, uplo, diag, dt)
        b0 = (rng.standard_normal(ldb * n) + (1j * rng.standard_normal(ldb * n) if cx else 0)).astype(dt)
        alpha = (0.75 - 0.5j) if cx else 0.75
        b = b0.copy()
        (complex3 if cx else level3).trmm(side, uplo, trans, diag, m, n, alpha, a, lda, b, ldb)
        B0 = b0.reshape(n, ldb).T[:m, :].astype(np.complex128 if cx else np.float64)
        opA = _dense_op(a.astype(np.complex128 if cx else np.float64), lda, q, mask, diag, trans)
        ref = alpha * (opA @ B0 if side == 0 else B0 @ opA)
        got = b.reshape(n, ldb).T[:m, :]
        den = abs(alpha) * np.linalg.norm(opA) * np.linalg.norm(B0)
        assert np.linalg.norm(got.astype(np.complex128) - ref) <= 4 * q * _u(dt) * den, (diag,)
        assert np.array_equal(b.reshape(n, ldb).T[m:, :], b0.reshape(n, ldb).T[m:, :])


def test_trmm_known_answer_and_alpha_zero():
    a = np.array([1.0, 0.0, 2.0, 3.0])  # [[1, 2], [0, 3]] column-major, upper
    b = np.array([1.0, 0.0, 0.0, 1.0])
    level3.trmm(0, 0, 0, 0, 2, 2, 1.0, a, 2, b, 2)
    assert list(b) == [1.0, 0.0, 2.0, 3.0]
    b = np.full(4, np.nan)
    level3.trmm(0, 0, 0, 0, 2, 2, 0.0, a, 2, b, 2)
    assert list(b) == [0.0] * 4


def test_trmm_argument_checks():
    with pytest.raises(InvalidLeadingDim):
        level3.trmm(0, 0, 0, 0, 4, 3, 1.0, np.zeros(16), 3, np.zeros(12), 4)
