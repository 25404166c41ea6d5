"""GPU parity tests of the rest of the Level-3 surface (complex GEMM, syrk,
symm, hemm, trsm), called through the C ABI and checked against the oracle:
the reference's own test assertions, then the restatement of rblas's
routines on the same seeded inputs.

Tolerances: GEMM-shaped results use the normwise bound 4*k*u (k the inner
dimension; for complex 4M/1M, u of the real type); trsm results (well
conditioned, diagonal in [1, 2], off-diagonal entries U[-0.1, 0.1]/order)
use a componentwise relative bound of 1e3*u on the solution and the
normwise backward error bound 4*q*u (q the triangle's order).
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
import rblas_b200 as rb
from rblas_b200 import complex3, level3
from rblas_b200.types import Precision
from tests.golden_runner import load_cases, run_case

pytestmark = pytest.mark.gpu

CASES = load_cases()


class GpuBackend:
    def gemm(self, layout, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
        level3.gemm(layout, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)

    def cgemm(self, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
        complex3.gemm(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)

    def syrk(self, *args):
        level3.syrk(*args)

    def symm(self, side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc):
        if np.iscomplexobj(c):
            complex3.symm(side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc)
        else:
            level3.symm(side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc)

    def hemm(self, *args):
        complex3.hemm(*args)

    def trsm(self, side, uplo, trans, diag, m, n, alpha, a, lda, b, ldb):
        if np.iscomplexobj(b):
            complex3.trsm(side, uplo, trans, diag, m, n, alpha, a, lda, b, ldb)
        else:
            level3.trsm(side, uplo, trans, diag, m, n, alpha, a, lda, b, ldb)


OPS = {"syrk", "symm", "trsm", "cgemm", "hemm", "ctrsm"}


@pytest.mark.parametrize("name", sorted(n for n, (m, _) in CASES.items() if m["op"] in OPS))
def test_reference_test_cases_on_gpu(name):
    meta, data = CASES[name]
    ok, detail = run_case(GpuBackend(), meta, data)
    assert ok, f"{name} ({meta['ref']}): {detail}"


def crand(rng, shape, dtype):
    return (rng.uniform(-1, 1, shape) + 1j * rng.uniform(-1, 1, shape)).astype(dtype)


def cnorm(x):
    return float(np.linalg.norm(np.asarray(x, dtype=np.complex128)))


def _u(dtype):
    return 2.0 ** -24 if np.dtype(dtype) in (np.float32, np.complex64) else 2.0 ** -53


# --------------------------------------------------------------------------
# complex GEMM
# --------------------------------------------------------------------------

@pytest.mark.parametrize("dtype", [np.complex64, np.complex128])
@pytest.mark.parametrize("ta", [0, 1, 2])
@pytest.mark.parametrize("tb", [0, 1, 2])
def test_complex_gemm_parity(dtype, ta, tb):
    rng = np.random.default_rng(10 * ta + tb)
    for (m, n, k) in [(1, 1, 1), (17, 13, 19), (65, 70, 131), (200, 96, 300)]:
        ar, ac = (k, m) if ta else (m, k)
        br, bc = (n, k) if tb else (k, n)
        A = crand(rng, (ac, ar), dtype)  # [col][row] -> flat col-major
        B = crand(rng, (bc, br), dtype)
        C0 = crand(rng, (n, m), dtype)
        a, b = A.reshape(-1), B.reshape(-1)
        alpha, beta = 1.0 + 0.5j, -0.25 + 0.75j
        c = C0.reshape(-1).copy()
        complex3.gemm(ta, tb, m, n, k, alpha, a, ar, b, br, beta, c, m)
        ref = C0.reshape(-1).copy()
        oracle.gemm(1, ta, tb, m, n, k, alpha, a, ar, b, br, beta, ref, m)
        den = abs(alpha) * cnorm(a) * cnorm(b) + abs(beta) * cnorm(C0)
        err = cnorm(c.astype(np.complex128) - ref) / den
        assert err <= 4 * k * _u(dtype), f"{(m, n, k)} {err:.3e}"


@pytest.mark.parametrize("dtype,prec", [(np.complex64, Precision.Bf16x6), (np.complex64, Precision.Bf16x3),
                                        (np.complex128, Precision.Ozaki)])
def test_complex_gemm_precision_forms(dtype, prec):
    """C32 through the BF16 split forms and C64 through Ozaki, ConjTrans x
    NoTrans, against the double-double oracle."""
    rng = np.random.default_rng(5)
    m, n, k = 160, 144, 512
    A = crand(rng, (m, k), dtype)  # stored k x m col-major: flat [i][p]
    B = crand(rng, (n, k), dtype)  # stored k x n
    a, b = A.reshape(-1), B.reshape(-1)
    alpha, beta = 1.0 + 0.5j, 0.0
    c = np.zeros(m * n, dtype)
    complex3.gemm(2, 0, m, n, k, alpha, a, k, b, k, beta, c, m, prec=prec)
    opA = np.conj(A.astype(np.complex128))           # op(A)[i, p]
    opB = B.astype(np.complex128).T                  # op(B)[p, j]
    hi, _ = oracle.dd_complex_gemm(opA, opB, alpha, 0.0)
    got = c.reshape(n, m).T
    den = abs(alpha) * cnorm(A) * cnorm(B)
    err = cnorm(got - hi) / den
    plain = np.zeros(m * n, dtype)
    complex3.gemm(2, 0, m, n, k, alpha, a, k, b, k, beta, plain, m)
    err_plain = cnorm(plain.reshape(n, m).T - hi) / den
    bound = 2 * err_plain + 2 * _u(dtype) if prec != Precision.Bf16x3 else 2.0 ** -15
    assert err <= bound, (err, err_plain)


def test_complex_gemm_beta_zero_ignores_nan():
    rng = np.random.default_rng(6)
    m, n, k = 30, 20, 25
    a = crand(rng, m * k, np.complex128)
    b = crand(rng, k * n, np.complex128)
    c = np.full(m * n, np.nan + 1j * np.nan)
    complex3.gemm(0, 0, m, n, k, 1.0, a, m, b, k, 0.0, c, m)
    assert not np.any(np.isnan(c))


# --------------------------------------------------------------------------
# syrk
# --------------------------------------------------------------------------

@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("uplo", [0, 1])
@pytest.mark.parametrize("trans", [0, 1])
def test_syrk_parity(dtype, uplo, trans):
    rng = np.random.default_rng(20 + 2 * uplo + trans)
    # n = 1000: the f32 product runs the narrow 128 x 64 tile under the triangle mask
    for (n, k, alpha, beta) in [(9, 11, 2.0, 3.0), (130, 77, 1.0, 0.0), (300, 257, -0.5, 1.0), (1000, 96, 1.5, -0.5)]:
        ar, ac = (k, n) if trans else (n, k)
        a = rng.uniform(-1, 1, ar * ac).astype(dtype)
        c0 = rng.uniform(-1, 1, n * n).astype(dtype)
        c = c0.copy()
        level3.syrk(uplo, trans, n, k, alpha, a, ar, beta, c, n)
        ref = c0.copy()
        oracle.syrk(uplo, trans, n, k, alpha, a, ar, beta, ref, n)
        G, R, C0 = c.reshape(n, n).T, ref.reshape(n, n).T, c0.reshape(n, n).T
        mask = np.triu(np.ones((n, n), bool)) if uplo == 0 else np.tril(np.ones((n, n), bool))
        assert np.array_equal(G[~mask], C0[~mask]), "other triangle modified"
        den = abs(alpha) * np.linalg.norm(a.astype(np.float64)) ** 2 + abs(beta) * np.linalg.norm(C0[mask])
        err = np.linalg.norm((G[mask].astype(np.float64) - R[mask])) / den
        assert err <= 4 * k * _u(dtype), (n, k, err)


# --------------------------------------------------------------------------
# symm / complex symm / hemm
# --------------------------------------------------------------------------

@pytest.mark.parametrize("dtype", [np.float32, np.float64, np.complex64, np.complex128])
@pytest.mark.parametrize("side", [0, 1])
@pytest.mark.parametrize("uplo", [0, 1])
def test_symm_parity(dtype, side, uplo):
    rng = np.random.default_rng(30 + 2 * side + uplo)
    cx = np.issubdtype(np.dtype(dtype), np.complexfloating)
    gen = (lambda s: crand(rng, s, dtype)) if cx else (lambda s: rng.uniform(-1, 1, s).astype(dtype))
    for (m, n) in [(2, 2), (37, 23), (150, 90)]:
        q = m if side == 0 else n
        a = gen(q * q)
        b = gen(m * n)
        c0 = gen(m * n)
        alpha, beta = (1.5 - 0.5j, 0.25 + 1j) if cx else (1.5, -0.75)
        for herm in ([False, True] if cx else [False]):
            c = c0.copy()
            ref = c0.copy()
            if herm:
                complex3.hemm(side, uplo, m, n, alpha, a, q, b, m, beta, c, m)
                oracle.hemm(side, uplo, m, n, alpha, a, q, b, m, beta, ref, m)
            elif cx:
                complex3.symm(side, uplo, m, n, alpha, a, q, b, m, beta, c, m)
                oracle.symm(side, uplo, m, n, alpha, a, q, b, m, beta, ref, m)
            else:
                level3.symm(side, uplo, m, n, alpha, a, q, b, m, beta, c, m)
                oracle.symm(side, uplo, m, n, alpha, a, q, b, m, beta, ref, m)
            den = abs(alpha) * cnorm(a) * cnorm(b) + abs(beta) * cnorm(c0)
            err = cnorm(c.astype(np.complex128) - ref) / den
            assert err <= 4 * q * _u(dtype), ((m, n), herm, err)


# --------------------------------------------------------------------------
# trsm
# --------------------------------------------------------------------------

def tri_matrix(rng, q, uplo, dtype):
    cx = np.issubdtype(np.dtype(dtype), np.complexfloating)
    off = rng.uniform(-0.1, 0.1, (q, q)) / max(1, q) ** 0.5
    if cx:
        off = off + 1j * rng.uniform(-0.1, 0.1, (q, q)) / max(1, q) ** 0.5
    A = np.tril(off, -1) if uplo == 1 else np.triu(off, 1)
    A = A + np.diag(rng.uniform(1, 2, q))
    junk = rng.uniform(-5, 5, (q, q))  # the other triangle is never referenced
    A = A + (np.triu(junk, 1) if uplo == 1 else np.tril(junk, -1))
    return np.asfortranarray(A.astype(dtype)).reshape(-1, order="F")


@pytest.mark.parametrize("dtype", [np.float32, np.float64, np.complex64, np.complex128])
@pytest.mark.parametrize("side", [0, 1])
@pytest.mark.parametrize("uplo", [0, 1])
@pytest.mark.parametrize("trans", [0, 1, 2])
def test_trsm_parity(dtype, side, uplo, trans):
    cx = np.issubdtype(np.dtype(dtype), np.complexfloating)
    if trans == 2 and not cx:
        pytest.skip("ConjTrans == Trans for real types")
    rng = np.random.default_rng(40 + 6 * side + 3 * uplo + trans)
    for (m, n) in [(3, 1), (70, 33), (150, 41)]:
        for diag in (0, 1):
            q = m if side == 0 else n
            a = tri_matrix(rng, q, uplo, dtype)
            b0 = (rng.uniform(-1, 1, m * n) + (1j * rng.uniform(-1, 1, m * n) if cx else 0)).astype(dtype)
            alpha = (0.75 + 0.25j) if cx else 0.75
            b = b0.copy()
            ref = b0.copy()
            if cx:
                complex3.trsm(side, uplo, trans, diag, m, n, alpha, a, q, b, m)
            else:
                level3.trsm(side, uplo, trans, diag, m, n, alpha, a, q, b, m)
            oracle.trsm(side, uplo, trans, diag, m, n, alpha, a, q, ref, m)
            rel = np.max(np.abs(b.astype(np.complex128) - ref)) / max(np.max(np.abs(ref)), 1e-30)
            assert rel <= 1e3 * _u(dtype), ((m, n), diag, rel)
            # normwise backward error of the GPU solution, which a wrong-order
            # update would push far past the bound even where the forward
            # error stays small
            back = _trsm_backward_error(a, b, b0, alpha, side, uplo, trans, diag, m, n, q)
            assert back <= 4 * q * _u(dtype), ((m, n), diag, back)
    assert rb.device_error()[0] == 0


def _trsm_backward_error(a, x, b0, alpha, side, uplo, trans, diag, m, n, q):
    """||op(A) X - alpha B||_F / (||A_tri||_F ||X||_F + |alpha| ||B||_F) in
    complex128, for trans 0 (NoTrans), 1 (Trans) or 2 (ConjTrans)."""
    A = a.reshape(q, q, order="F").astype(np.complex128)
    T = np.tril(A) if uplo == 1 else np.triu(A)
    if diag == 1:
        np.fill_diagonal(T, 1.0)
    opA = T if trans == 0 else (T.T if trans == 1 else T.conj().T)
    X = x.reshape(m, n, order="F").astype(np.complex128)
    B0 = b0.reshape(m, n, order="F").astype(np.complex128)
    R = (opA @ X if side == 0 else X @ opA) - alpha * B0
    return np.linalg.norm(R) / (np.linalg.norm(T) * np.linalg.norm(X) + abs(alpha) * np.linalg.norm(B0))


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("side", [0, 1])
@pytest.mark.parametrize("uplo", [0, 1])
@pytest.mark.parametrize("trans", [0, 1])
def test_trsm_blocked_parity(dtype, side, uplo, trans):
    """Orders above one 512-row diagonal block (1100: two full blocks and a
    ragged 76-row one), so the real types' blocked path runs its GEMM
    updates between the diagonal solves. Forward error as in
    test_trsm_parity, and the normwise backward error
    ||op(A) X - alpha B||_F / (||A_tri||_F ||X||_F + |alpha| ||B||_F) within
    4 * q * u."""
    rng = np.random.default_rng(70 + 4 * side + 2 * uplo + trans)
    q, nr = 1100, 70
    m, n = (q, nr) if side == 0 else (nr, q)
    for diag in (0, 1):
        a = tri_matrix(rng, q, uplo, dtype)
        b0 = rng.uniform(-1, 1, m * n).astype(dtype)
        b = b0.copy()
        ref = b0.copy()
        level3.trsm(side, uplo, trans, diag, m, n, 0.75, a, q, b, m)
        oracle.trsm(side, uplo, trans, diag, m, n, 0.75, a, q, ref, m)
        rel = np.max(np.abs(b.astype(np.float64) - ref)) / np.max(np.abs(ref))
        assert rel <= 1e3 * _u(dtype), (diag, rel)
        A = a.reshape(q, q, order="F").astype(np.float64)
        T = np.tril(A) if uplo == 1 else np.triu(A)
        if diag == 1:
            np.fill_diagonal(T, 1.0)
        opA = T.T if trans else T
        X = b.reshape(m, n, order="F").astype(np.float64)
        B0 = b0.reshape(m, n, order="F").astype(np.float64)
        R = (opA @ X if side == 0 else X @ opA) - 0.75 * B0
        back = np.linalg.norm(R) / (np.linalg.norm(T) * np.linalg.norm(X) + 0.75 * np.linalg.norm(B0))
        assert back <= 4 * q * _u(dtype), (diag, back)
    assert rb.device_error()[0] == 0


def test_trsm_alpha_zero_and_unit_diag_ignore_diagonal():
    rng = np.random.default_rng(50)
    for m, n in [(40, 9), (600, 9)]:  # one diagonal block; two (the blocked path)
        a = tri_matrix(rng, m, 1, np.float64)
        A = a.reshape(m, m, order="F")
        A[np.diag_indices(m)] = np.nan  # Unit: the diagonal is never read
        b = rng.uniform(-1, 1, m * n)
        ref = b.copy()
        level3.trsm(0, 1, 0, 1, m, n, 1.0, a, m, b, m)
        oracle.trsm(0, 1, 0, 1, m, n, 1.0, a, m, ref, m)
        assert np.max(np.abs(b - ref)) < 1e-12, m
