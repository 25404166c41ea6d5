"""GPU tests of the pipelined host path of symm / hemm, syrk, trsm and trmm: calls
of at least 64 MB upload A once and run independent panels of B (and C) --
columns for side Left, rows for Right -- on their own streams. Checked
against dense float64 / complex128 numpy evaluations: symm and trmm within
the normwise bound 4*q*u of |alpha| ||op(A)|| ||B|| (+ |beta| ||C||), syrk
within 4*k*u of |alpha| ||A||^2 + |beta| ||C_tri||, trsm by
the normwise backward error ||op(A) X - alpha B|| / (||A_tri|| ||X|| +
|alpha| ||B||) within 4*q*u, and for the real trsm / trmm also against the
device-pointer call on the same operands (which runs unsplit). Padded
leading dimensions: rows beyond m stay untouched."""
from __future__ import annotations

import numpy as np
import pytest

import rblas_b200 as rb
from rblas_b200 import complex3, level3

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _u(dt):
    return 2.0 ** -24 if np.dtype(dt) in (np.float32, np.complex64) else 2.0 ** -53


def _gen(rng, shape, dt):
    x = rng.uniform(-1, 1, shape)
    if np.issubdtype(np.dtype(dt), np.complexfloating):
        x = x + 1j * rng.uniform(-1, 1, shape)
    return x.astype(dt)


def _tri(rng, q, uplo, dt):
    """Well-conditioned triangle (diagonal in [1, 2]) with junk in the other one."""
    off = _gen(rng, (q, q), dt) * (0.1 / q ** 0.5)
    T = (np.tril(off, -1) if uplo == 1 else np.triu(off, 1)) + np.diag(rng.uniform(1, 2, q))
    junk = _gen(rng, (q, q), dt) * 5
    full = T + (np.triu(junk, 1) if uplo == 1 else np.tril(junk, -1))
    return np.asfortranarray(full.astype(dt)), T.astype(np.complex128 if np.iscomplexobj(full) else np.float64)


# (side, m, n): Left splits B's 1024 (768) columns, Right its rows
SHAPES = [(0, 2900, 1024), (1, 1024, 2900)]


@pytest.mark.parametrize("side,m,n", SHAPES)
@pytest.mark.parametrize("uplo,trans", [(1, 0), (0, 1)])
def test_trsm_host_panels(side, m, n, uplo, trans):
    rng = np.random.default_rng(300 + 7 * side + 2 * uplo + trans)
    q = m if side == 0 else n
    A, T = _tri(rng, q, uplo, np.float64)
    ldb = m + 3
    b0 = rng.uniform(-1, 1, (n, ldb)).T.copy(order="F")  # ldb x n, column-major
    b = b0.copy(order="F")
    level3.trsm(side, uplo, trans, 0, m, n, 0.5, A.reshape(-1, order="F"), q, b.reshape(-1, order="F"), ldb)
    X = b[:m, :]
    assert np.array_equal(b[m:, :], b0[m:, :])
    opA = T.T if trans else T
    R = (opA @ X if side == 0 else X @ opA) - 0.5 * b0[:m, :]
    back = np.linalg.norm(R) / (np.linalg.norm(T) * np.linalg.norm(X) + 0.5 * np.linalg.norm(b0[:m, :]))
    assert back <= 4 * q * _u(np.float64), back
    # the device-pointer call (one piece) on the same operands
    A_d = torch.tensor(A.reshape(-1, order="F"), device="cuda")
    B_d = torch.tensor(b0.reshape(-1, order="F"), device="cuda")
    level3.trsm_dev(side, uplo, trans, 0, m, n, 0.5, A_d.data_ptr(), q, B_d.data_ptr(), ldb)
    torch.cuda.synchronize()
    Xd = B_d.cpu().numpy().reshape(ldb, n, order="F")[:m, :]
    assert np.max(np.abs(Xd - X)) <= 1e3 * _u(np.float64) * np.max(np.abs(X))
    assert rb.device_error()[0] == 0


@pytest.mark.parametrize("side,m,n", SHAPES)
@pytest.mark.parametrize("uplo,trans,diag", [(1, 0, 0), (0, 1, 1)])
def test_trmm_host_panels(side, m, n, uplo, trans, diag):
    rng = np.random.default_rng(400 + 7 * side + 2 * uplo + trans)
    q = m if side == 0 else n
    A, T = _tri(rng, q, uplo, np.float64)
    if diag == 1:
        np.fill_diagonal(T, 1.0)
    ldb = m + 3
    b0 = rng.uniform(-1, 1, (n, ldb)).T.copy(order="F")
    b = b0.copy(order="F")
    level3.trmm(side, uplo, trans, diag, m, n, 0.75, A.reshape(-1, order="F"), q, b.reshape(-1, order="F"), ldb)
    assert np.array_equal(b[m:, :], b0[m:, :])
    opA = T.T if trans else T
    ref = 0.75 * (opA @ b0[:m, :] if side == 0 else b0[:m, :] @ opA)
    den = 0.75 * np.linalg.norm(opA) * np.linalg.norm(b0[:m, :])
    assert np.linalg.norm(b[:m, :] - ref) <= 4 * q * _u(np.float64) * den
    assert rb.device_error()[0] == 0


@pytest.mark.parametrize("dt", [np.float64, np.complex128])
@pytest.mark.parametrize("side,m,n", [(0, 2900, 1024), (1, 1024, 2900)])
@pytest.mark.parametrize("beta", [0.0, -0.5])
def test_symm_host_panels(dt, side, m, n, beta):
    cx = np.issubdtype(np.dtype(dt), np.complexfloating)
    if cx:  # complex128 operands are twice the bytes: smaller orders still reach the split
        m, n = (2048, 768) if side == 0 else (768, 2048)
    rng = np.random.default_rng(500 + side + (2 if cx else 0))
    q = m if side == 0 else n
    A = _gen(rng, (q, q), dt)
    lower = np.tril(A)
    S = lower + np.tril(A, -1).T  # symmetric from the lower triangle (junk above is never read)
    ldb, ldc = m + 1, m + 2
    B = np.asfortranarray(_gen(rng, (ldb, n), dt))
    C0 = np.asfortranarray(_gen(rng, (ldc, n), dt))
    c = C0.copy(order="F")
    alpha = (0.5 + 0.25j) if cx else 0.5
    args = (side, 1, m, n, alpha, np.asfortranarray(A).reshape(-1, order="F"), q, B.reshape(-1, order="F"), ldb,
            beta, c.reshape(-1, order="F"), ldc)
    (complex3 if cx else level3).symm(*args)
    opS = S.astype(np.complex128 if cx else np.float64)
    Bm = B[:m, :]
    ref = alpha * (opS @ Bm if side == 0 else Bm @ opS) + beta * C0[:m, :]
    den = abs(alpha) * np.linalg.norm(opS) * np.linalg.norm(Bm) + abs(beta) * np.linalg.norm(C0[:m, :])
    assert np.linalg.norm(c[:m, :] - ref) <= 4 * q * _u(dt) * den
    assert np.array_equal(c[m:, :], C0[m:, :])
    assert rb.device_error()[0] == 0


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("uplo", [0, 1])
@pytest.mark.parametrize("trans", [0, 1])
def test_syrk_host_panels(dt, uplo, trans):
    """Column panels of C: the lower triangle's panel is one masked product
    from the diagonal down, the upper's a plain product above a masked
    diagonal block; the other triangle comes back unchanged."""
    rng = np.random.default_rng(600 + 2 * uplo + trans)
    n, k = 3000, 1000
    ar, ac = (k, n) if trans else (n, k)
    lda, ldc = ar + 1, n + 2
    A = np.asfortranarray(rng.uniform(-1, 1, (lda, ac)).astype(dt))
    C0 = np.asfortranarray(rng.uniform(-1, 1, (ldc, n)).astype(dt))
    c = C0.copy(order="F")
    level3.syrk(uplo, trans, n, k, 1.5, A.reshape(-1, order="F"), lda, -0.5, c.reshape(-1, order="F"), ldc)
    opA = (A[:ar, :].T if trans else A[:ar, :]).astype(np.float64)
    ref = 1.5 * opA @ opA.T - 0.5 * C0[:n, :].astype(np.float64)
    mask = np.triu(np.ones((n, n), bool)) if uplo == 0 else np.tril(np.ones((n, n), bool))
    got = c[:n, :]
    assert np.array_equal(got[~mask], C0[:n, :][~mask]), "other triangle modified"
    assert np.array_equal(c[n:, :], C0[n:, :])
    den = 1.5 * np.linalg.norm(opA) ** 2 + 0.5 * np.linalg.norm(C0[:n, :][mask])
    assert np.linalg.norm(got[mask].astype(np.float64) - ref[mask]) <= 4 * k * _u(dt) * den
    assert rb.device_error()[0] == 0
