"""CPU tests of the oracle itself: it must satisfy every assertion of the
reference's own test suite (the golden cases) before the GPU library's
parity tests compare against it."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from tests.golden_runner import load_cases, run_case

CASES = load_cases()


class OracleBackend:
    def gemm(self, layout, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
        oracle.gemm(layout, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)

    def cgemm(self, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
        oracle.gemm(1, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)

    def syrk(self, *args):
        oracle.syrk(*args)

    def symm(self, *args):
        oracle.symm(*args)

    def hemm(self, *args):
        oracle.hemm(*args)

    def trsm(self, *args):
        oracle.trsm(*args)

    def check_gemm(self, *args):
        rc, err = oracle.check_gemm(*args)
        which = err.which.decode() if err.which else ""
        return rc, which, err.got, err.min_or_need


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_meets_reference_assertions(name):
    meta, data = CASES[name]
    ok, detail = run_case(OracleBackend(), meta, data)
    assert ok, f"{name} ({meta['ref']}): {detail}"


@pytest.mark.parametrize("name", ["gemm_matches_reference", "correctness_large_random_sgemm"])
def test_oracle_scalar_fallback_meets_assertions(name):
    """The no-AVX2 microkernel (src/kernel/gemm.rs:641-670) passes too."""
    meta, data = CASES[name]
    oracle.set_force_scalar(True)
    try:
        ok, detail = run_case(OracleBackend(), meta, data)
    finally:
        oracle.set_force_scalar(False)
    assert ok, detail


def test_complex_mul_kat():
    # src/complex.rs:122-130: (1+2i)(3-i) = 5+5i exactly
    a = np.array([1 + 2j], dtype=np.complex128)
    b = np.array([3 - 1j], dtype=np.complex128)
    c = np.zeros(1, dtype=np.complex128)
    oracle.gemm(1, 0, 0, 1, 1, 1, 1.0, a, 1, b, 1, 0.0, c, 1)
    assert c[0] == 5 + 5j


def test_avx2_vs_scalar_microkernel_close():
    """src/kernel/gemm.rs:724-770: AVX2 tile agrees with the scalar tile."""
    rng = np.random.default_rng(1)
    m, n, k = 37, 29, 531  # crosses KC=512 and MR/NR edges
    a = rng.uniform(-1, 1, m * k).astype(np.float32)
    b = rng.uniform(-1, 1, k * n).astype(np.float32)
    c1 = rng.uniform(-1, 1, m * n).astype(np.float32)
    c2 = c1.copy()
    oracle.gemm(1, 0, 0, m, n, k, 1.5, a, m, b, k, 0.5, c1, m, threads=1)
    oracle.set_force_scalar(True)
    try:
        oracle.gemm(1, 0, 0, m, n, k, 1.5, a, m, b, k, 0.5, c2, m, threads=1)
    finally:
        oracle.set_force_scalar(False)
    assert np.max(np.abs(c1 - c2)) < 1e-4


def test_threaded_equals_serial_within_tolerance():
    """gemm_parallel changes only full/edge writeback at chunk ends."""
    rng = np.random.default_rng(2)
    m, n, k = 64, 700, 48
    a = rng.uniform(-1, 1, m * k).astype(np.float32)
    b = rng.uniform(-1, 1, k * n).astype(np.float32)
    c1 = np.zeros(m * n, np.float32)
    c2 = np.zeros(m * n, np.float32)
    oracle.gemm(1, 0, 0, m, n, k, 1.0, a, m, b, k, 0.0, c1, m, threads=1)
    oracle.gemm(1, 0, 0, m, n, k, 1.0, a, m, b, k, 0.0, c2, m, threads=4)
    assert np.max(np.abs(c1 - c2)) < 1e-5


def test_beta_zero_does_not_read_c():
    """apply_beta (src/kernel/gemm.rs:322-338): beta == 0 writes zeros, so NaN in C0 vanishes."""
    m = n = k = 5
    a = np.ones(m * k, np.float64)
    b = np.ones(k * n, np.float64)
    c = np.full(m * n, np.nan)
    oracle.gemm(1, 0, 0, m, n, k, 1.0, a, m, b, k, 0.0, c, m)
    assert np.all(c == k)


def test_k_zero_and_alpha_zero_only_scale_c():
    m, n = 4, 3
    a = np.ones(m * 2)
    b = np.ones(2 * n)
    c = np.arange(m * n, dtype=np.float64)
    oracle.gemm(1, 0, 0, m, n, 0, 1.0, a, m, b, 1, 2.0, c, m)
    assert np.array_equal(c, 2 * np.arange(m * n))
    c = np.arange(m * n, dtype=np.float64)
    oracle.gemm(1, 0, 0, m, n, 2, 0.0, a, m, b, 2, 0.5, c, m)
    assert np.array_equal(c, 0.5 * np.arange(m * n))


def test_row_major_all_transposes_match_numpy():
    rng = np.random.default_rng(3)
    m, n, k = 23, 17, 31
    for ta in (0, 1):
        for tb in (0, 1):
            A = rng.standard_normal((k, m) if ta else (m, k))
            B = rng.standard_normal((n, k) if tb else (k, n))
            C0 = rng.standard_normal((m, n))
            c = C0.reshape(-1).copy()
            oracle.gemm(0, ta, tb, m, n, k, 1.5, A.reshape(-1), A.shape[1], B.reshape(-1),
                        B.shape[1], -0.5, c, n)
            want = 1.5 * (A.T if ta else A) @ (B.T if tb else B) - 0.5 * C0
            assert np.max(np.abs(c.reshape(m, n) - want)) < 1e-12


def test_dd_oracle_exact_on_integers():
    """Integer inputs with exact products: the dd result equals exact math."""
    rng = np.random.default_rng(4)
    m, n, k = 9, 7, 64
    A = rng.integers(-2 ** 20, 2 ** 20, (m, k)).astype(np.float64)
    B = rng.integers(-2 ** 20, 2 ** 20, (k, n)).astype(np.float64)
    hi, lo = oracle.dd_gemm(0, 0, 0, m, n, k, 1.0, A.reshape(-1), k, B.reshape(-1), n, 0.0, None, n)
    exact = [[sum(int(A[i, p]) * int(B[p, j]) for p in range(k)) for j in range(n)] for i in range(m)]
    for i in range(m):
        for j in range(n):
            assert int(hi[i, j]) + int(lo[i, j]) == exact[i][j]


def test_dd_oracle_row_sample_matches_full():
    rng = np.random.default_rng(5)
    m, n, k = 40, 12, 33
    a = rng.standard_normal(m * k)
    b = rng.standard_normal(k * n)
    c0 = rng.standard_normal(m * n)
    hi, lo = oracle.dd_gemm(1, 0, 0, m, n, k, 1.5, a, m, b, k, -0.5, c0, m)
    rows = np.array([0, 7, 39, 20])
    hs, ls = oracle.dd_gemm(1, 0, 0, m, n, k, 1.5, a, m, b, k, -0.5, c0, m, rows=rows)
    assert np.array_equal(hs, hi[rows]) and np.array_equal(ls, lo[rows])


def test_restatement_error_within_4ku_of_dd_oracle():
    """The stated tolerance ||C-Cref||_F/(|a|||A|| ||B|| + |b| ||C0||) <= 4 k u
    holds for the restatement itself (f32, 1024^3-like shape scaled down)."""
    rng = np.random.default_rng(6)
    m, n, k = 128, 96, 700
    a = rng.uniform(-1, 1, m * k).astype(np.float32)
    b = rng.uniform(-1, 1, k * n).astype(np.float32)
    c = np.zeros(m * n, np.float32)
    oracle.gemm(1, 0, 0, m, n, k, 1.0, a, m, b, k, 0.0, c, m)
    hi, lo = oracle.dd_gemm(1, 0, 0, m, n, k, 1.0, a, m, b, k, 0.0, None, m)
    err = oracle.normwise_error(c.reshape(n, m).T, hi, lo, 1.0, np.linalg.norm(a.astype(np.float64)),
                                np.linalg.norm(b.astype(np.float64)), 0.0, 0.0)
    assert err <= 4 * k * 2.0 ** -24
