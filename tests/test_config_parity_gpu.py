"""Parity at the full configuration sizes of the real and complex GEMM
workloads, through the host API (rblas's slice-based calls), against the
restatement of rblas's gemm (oracle.gemm: level3::gemm src/level3.rs:32-62,
kernel/gemm.rs, gemm_avx2.rs; complex3::gemm src/complex3.rs:27-125) on the
same seeded inputs and against the double-double oracle on a seeded row
sample.

Tolerances (normwise ||C - C_ref||_F / (|alpha| ||A||_F ||B||_F + |beta| ||C0||_F),
u of the real type):
  * plain forms: <= 4*k*u against the restatement and against the oracle;
  * OZAKI and BF16X6: <= 4*k*u against the oracle and <= 2 x the plain
    form's own error on the same inputs + 2u (u/16 for the row-sampled
    real cases);
  * BF16X3: <= 2^-15 (three bf16 products keep ~16 significand bits).
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from rblas_b200 import complex3, level3
from rblas_b200.types import Layout, Precision
from tests.util import Problem

pytestmark = pytest.mark.gpu


def run(p: Problem, prec):
    c = p.fresh_c()
    level3.gemm(p.layout, p.ta, p.tb, p.m, p.n, p.k, p.alpha, p.a, p.lda, p.b, p.ldb, p.beta, c, p.ldc,
                prec=prec)
    return c


@pytest.mark.parametrize("dist", ["normal", "pow2"])
def test_dgemm_3000x5000x2048_rowmajor_plain_and_ozaki(dist):
    """The non-square DGEMM case: f64 row-major N/N, alpha = 1.5, beta = -0.5;
    standard normal entries and the sign*2^e set (e uniform in [-30, 30])."""
    p = Problem(Layout.RowMajor, 0, 0, 3000, 5000, 2048, np.float64, alpha=1.5, beta=-0.5, seed=41, dist=dist)
    ref = p.reference_restatement()
    plain = run(p, Precision.Plain)
    oz = run(p, Precision.Ozaki)
    assert p.normwise(plain, ref) <= p.tol()
    assert p.normwise(oz, ref) <= p.tol()
    rows = np.sort(np.random.default_rng(42).choice(p.m, 64, replace=False))
    e_pl = p.normwise_vs_dd(plain, rows=rows)
    e_oz = p.normwise_vs_dd(oz, rows=rows)
    assert e_pl <= p.tol() and e_oz <= p.tol(), (e_pl, e_oz)
    assert e_oz <= 2 * e_pl + 2.0 ** -57, (e_oz, e_pl)


@pytest.mark.parametrize("ta,tb", [(0, 0), (1, 0), (0, 1), (1, 1)])
def test_plain_dgemm_4096_matches_restatement(ta, tb):
    """The square DGEMM case in the plain form (FP64 products on the FP64
    tensor cores): f64 row-major, all four transposes, alpha = 1.5,
    beta = -0.5, standard normal entries, against the restatement of rblas's
    gemm over the whole of C."""
    p = Problem(Layout.RowMajor, ta, tb, 4096, 4096, 4096, np.float64, alpha=1.5, beta=-0.5, seed=43 + 2 * ta + tb,
                dist="normal")
    ref = p.reference_restatement()
    err = p.normwise(run(p, Precision.Plain), ref)
    assert err <= p.tol(), (err, p.tol())


def _crand(rng, shape, dtype):
    return (rng.uniform(-1, 1, shape) + 1j * rng.uniform(-1, 1, shape)).astype(dtype)


def _cnorm(x):
    return float(np.linalg.norm(np.asarray(x, dtype=np.complex128)))


@pytest.mark.parametrize("dtype", [np.complex64, np.complex128])
def test_complex_2048_conjtrans_notrans_all_forms(dtype):
    """The complex case: ConjTrans x NoTrans, m = n = k = 2048,
    alpha = (1, 0.5), beta = (0, 0), real and imaginary parts uniform in
    [-1, 1). C64 runs plain FP64 and Ozaki; C32 runs plain FP32, BF16X3 and
    BF16X6."""
    m = n = k = 2048
    u = 2.0 ** -24 if dtype == np.complex64 else 2.0 ** -53
    rng = np.random.default_rng(44)
    A = _crand(rng, (m, k), dtype)  # flat [i][p]: stored k x m column-major
    B = _crand(rng, (n, k), dtype)  # stored k x n
    a, b = A.reshape(-1), B.reshape(-1)
    alpha, beta = 1.0 + 0.5j, 0.0
    den = abs(alpha) * _cnorm(A) * _cnorm(B)

    def call(prec):
        c = np.full(m * n, np.nan, dtype)  # beta == 0: C is never read
        complex3.gemm(2, 0, m, n, k, alpha, a, k, b, k, beta, c, m, prec=prec)
        return c

    plain = call(Precision.Plain)
    ref = np.zeros(m * n, dtype)
    oracle.gemm(1, 2, 0, m, n, k, alpha, a, k, b, k, beta, ref, m)
    assert _cnorm(plain.astype(np.complex128) - ref) / den <= 4 * k * u
    rows = np.sort(np.random.default_rng(45).choice(m, 64, replace=False))
    opA = np.conj(A[rows].astype(np.complex128))       # op(A)[i, p] on the sampled rows
    opB = B.astype(np.complex128).T                    # op(B)[p, j]
    hi, _ = oracle.dd_complex_gemm(opA, opB, alpha, 0.0)
    den_rows = abs(alpha) * _cnorm(A[rows]) * _cnorm(B)

    def err(c):
        return _cnorm(c.reshape(n, m).T[rows] - hi) / den_rows

    e_plain = err(plain)
    assert e_plain <= 4 * k * u
    forms = (Precision.Ozaki,) if dtype == np.complex128 else (Precision.Bf16x3, Precision.Bf16x6)
    for prec in forms:
        e = err(call(prec))
        if prec == Precision.Bf16x3:
            assert e <= 2.0 ** -15, e
        else:
            assert e <= 4 * k * u, (prec, e)
            assert e <= 2 * e_plain + 2 * u, (prec, e, e_plain)
