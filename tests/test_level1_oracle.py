"""The oracle's Level-1 restatement (level1::axpy / dot / scal / nrm2 / asum /
copy / swap, complex1::axpy / dotu / dotc / scal / nrm2) pinned on the
reference's own tests (src/level1.rs:169-234, src/complex1.rs:119-145), plus
strided forms against numpy and exact sums; and the library's Level-1
argument rules, which return before any device work (CPU only)."""
from __future__ import annotations

import math
from fractions import Fraction

import numpy as np
import pytest

import oracle
import rblas_b200 as rb
from rblas_b200 import complex1, level1


# ---- the reference's tests, on the oracle ---------------------------------------

def test_axpy_contiguous():  # src/level1.rs:169-175
    x = np.array([1.0, 2.0, 3.0, 4.0], dtype=np.float32)
    y = np.array([10.0, 20.0, 30.0, 40.0], dtype=np.float32)
    oracle.axpy(4, 2.0, x, 1, y, 1)
    assert list(y) == [12.0, 24.0, 36.0, 48.0]


def test_axpy_strided():  # src/level1.rs:177-183
    x = np.array([1.0, 0.0, 2.0, 0.0, 3.0])
    y = np.array([10.0, 20.0, 30.0])
    oracle.axpy(3, 1.0, x, 2, y, 1)
    assert list(y) == [11.0, 22.0, 33.0]


def test_dot_basic():  # src/level1.rs:185-190
    x = np.array([1.0, 2.0, 3.0], dtype=np.float32)
    y = np.array([4.0, 5.0, 6.0], dtype=np.float32)
    assert oracle.dot(3, x, 1, y, 1) == 32.0


def test_scal_basic():  # src/level1.rs:192-197
    x = np.array([1.0, 2.0, 3.0])
    oracle.scal(3, 10.0, x, 1)
    assert list(x) == [10.0, 20.0, 30.0]


def test_nrm2_basic():  # src/level1.rs:199-203
    assert abs(oracle.nrm2(2, np.array([3.0, 4.0], dtype=np.float32), 1) - 5.0) < 1e-6


def test_nrm2_no_overflow():  # src/level1.rs:205-215
    big = 1.0e200
    got = oracle.nrm2(3, np.array([big, big, big]), 1)
    assert math.isfinite(got)
    want = big * math.sqrt(3.0)
    assert abs(got - want) / want < 1e-12


def test_nrm2_matches_naive_for_moderate():  # src/level1.rs:217-222
    x = np.array([1.0, -2.0, 3.0, -4.0, 5.0])
    assert abs(oracle.nrm2(5, x, 1) - math.sqrt(float(np.sum(x * x)))) < 1e-12


def test_nrm2_strided():  # src/level1.rs:224-228
    assert abs(oracle.nrm2(2, np.array([3.0, 99.0, 4.0]), 2) - 5.0) < 1e-12


def test_asum_basic():  # src/level1.rs:230-234
    assert oracle.asum(4, np.array([1.0, -2.0, 3.0, -4.0]), 1) == 10.0


def test_complex_axpy_and_scal():  # src/complex1.rs:119-129
    x = np.array([1 + 1j, 2 - 1j])
    y = np.array([0 + 0j, 1 + 1j])
    oracle.axpy(2, 2 + 0j, x, 1, y, 1)
    assert list(y) == [2 + 2j, 5 - 1j]
    z = np.array([1 + 0j])
    oracle.scal(1, 0 + 1j, z, 1)
    assert list(z) == [1j]


def test_dotu_vs_dotc():  # src/complex1.rs:131-139
    x = np.array([1 + 2j])
    y = np.array([3 + 4j])
    assert oracle.dot(1, x, 1, y, 1) == -5 + 10j
    assert oracle.dot(1, x, 1, y, 1, conj=True) == 11 - 2j


def test_complex_nrm2_basic():  # src/complex1.rs:141-145
    assert abs(oracle.nrm2(1, np.array([3 + 4j]), 1) - 5.0) < 1e-12


# ---- strided forms and rounding -------------------------------------------------

def _exact_dot(x, y):
    return float(sum(Fraction(float(a)) * Fraction(float(b)) for a, b in zip(x, y)))


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("incx,incy", [(1, 1), (2, 3), (3, 1)])
def test_real_strided_against_numpy(dtype, incx, incy):
    rng = np.random.default_rng(11 + incx + 5 * incy)
    n = 203  # crosses the AVX2 blocks of 2W and W and leaves a tail
    x = rng.standard_normal(n * incx).astype(dtype)
    y0 = rng.standard_normal(n * incy).astype(dtype)
    xs, ys = x[::incx][:n], y0[::incy][:n]
    y = y0.copy()
    oracle.axpy(n, 0.75, x, incx, y, incy)
    want = y0.copy()
    want[::incy][:n] = [float(Fraction(0.75) * Fraction(float(a)) + Fraction(float(b))) for a, b in zip(xs, ys)]
    # one rounding of the exact alpha*x + y (fma), rounded again to the dtype
    assert np.array_equal(y, want.astype(dtype))
    eps = np.finfo(dtype).eps
    exact = _exact_dot(xs, ys)
    bound = n * eps * float(np.sum(np.abs(xs.astype(np.float64) * ys)))
    assert abs(oracle.dot(n, x, incx, y0, incy) - exact) <= bound
    assert abs(oracle.asum(n, x, incx) - float(np.sum(np.abs(xs.astype(np.float64))))) <= n * eps * 4 * n
    assert abs(oracle.nrm2(n, x, incx) - math.sqrt(float(np.sum(xs.astype(np.float64) ** 2)))) <= 4 * n * eps * 10
    s = x.copy()
    oracle.scal(n, -1.5, s, incx)
    w = x.copy()
    w[::incx][:n] = (np.float64(-1.5) * xs.astype(np.float64)).astype(dtype)
    assert np.array_equal(s, w)


def test_axpy_is_one_fused_rounding():
    """fma(alpha, x, y): alpha*x is not rounded on its own (src/kernel/avx2.rs:19)."""
    a = 1.0 + 2.0 ** -12
    x = np.array([a], dtype=np.float32)
    y = np.array([-1.0], dtype=np.float32)
    oracle.axpy(1, a, x, 1, y, 1)
    assert y[0] == np.float32(2.0 ** -11 + 2.0 ** -24)  # a*a rounded first would give 2^-11


def test_copy_and_swap_follow_the_loop():
    x = np.array([1.0, 2.0, 3.0])
    y = np.zeros(5)
    oracle.copy(3, x, 1, y, 2)
    assert list(y) == [1.0, 0.0, 2.0, 0.0, 3.0]
    y1 = np.zeros(1)
    oracle.copy(3, x, 1, y1, 0)  # every element lands on y[0]; the last stays
    assert y1[0] == 3.0
    a, b = np.array([1.0, 2.0]), np.array([3.0, 4.0])
    oracle.swap(2, a, 1, b, 1)
    assert list(a) == [3.0, 4.0] and list(b) == [1.0, 2.0]


def test_nrm2_scaling_edges():
    tiny = 1.0e-200
    assert abs(oracle.nrm2(4, np.full(4, tiny), 1) - 2 * tiny) / (2 * tiny) < 1e-12  # no underflow
    assert oracle.nrm2(3, np.zeros(3), 1) == 0.0
    assert math.isinf(oracle.nrm2(3, np.array([1.0, np.inf, 2.0]), 1))
    assert math.isnan(oracle.nrm2(2, np.array([np.inf, np.inf]), 1))  # inf/inf in the rescale
    assert math.isnan(oracle.nrm2(3, np.array([1.0, np.nan, 2.0]), 1))


# ---- the library's argument rules (no device work on these paths) ---------------

def test_zero_n_and_alpha_early_returns():
    x = np.ones(4)
    y = np.ones(4)
    level1.axpy(0, 2.0, x, 1, y, 1)
    level1.axpy(4, 0.0, x, 0, y, 0)  # alpha == 0 returns before the stride checks (src/level1.rs:18)
    level1.scal(4, 1.0, x, 0)        # alpha == 1 likewise (src/level1.rs:71)
    assert level1.dot(0, x, 1, y, 1) == 0.0
    assert level1.nrm2(0, x, 0) == 0.0
    assert level1.asum(0, x, 1) == 0.0
    assert complex1.dotu(0, np.ones(2, np.complex128), 1, np.ones(2, np.complex128), 1) == 0j
    assert complex1.nrm2(0, np.ones(2, np.complex64), 0) == 0.0
    assert list(x) == [1.0] * 4 and list(y) == [1.0] * 4


@pytest.mark.parametrize("call,which", [
    (lambda x, y: level1.axpy(3, 2.0, x, 0, y, 1), "x"),
    (lambda x, y: level1.axpy(3, 2.0, x, 1, y, 0), "y"),
    (lambda x, y: level1.dot(3, x, 2, y, 0), "y"),
    (lambda x, y: level1.scal(3, 2.0, x, 0), "x"),
    (lambda x, y: level1.nrm2(3, x, 0), "x"),
    (lambda x, y: level1.swap(3, x, 0, y, 1), "x"),
    (lambda x, y: complex1.axpy(2, 1j, x.astype(np.complex128), 0, y.astype(np.complex128), 1), "x"),
    (lambda x, y: complex1.scal(2, 1j, x.astype(np.complex64), 0), "x"),
    (lambda x, y: complex1.nrm2(2, x.astype(np.complex128), 0), "x"),
])
def test_zero_strides_where_rblas_asserts(call, which):
    with pytest.raises(rb.ZeroStride) as e:
        call(np.ones(8), np.ones(8))
    assert e.value.which == which


@pytest.mark.parametrize("call,which,got,need", [
    (lambda: level1.axpy(5, 2.0, np.ones(4), 1, np.ones(5), 1), "x", 4, 5),
    (lambda: level1.axpy(3, 2.0, np.ones(5), 2, np.ones(5), 3), "y", 5, 7),
    (lambda: level1.dot(4, np.ones(4), 1, np.ones(3), 1), "y", 3, 4),
    (lambda: level1.asum(3, np.ones(2), 0 + 1), "x", 2, 3),
    (lambda: level1.copy(3, np.ones(5), 2, np.ones(2), 1), "y", 2, 3),
    (lambda: complex1.dotc(3, np.ones(3, np.complex64), 1, np.ones(8, np.complex64), 4), "y", 8, 9),
])
def test_buffer_too_small(call, which, got, need):
    with pytest.raises(rb.BufferTooSmall) as e:
        call()
    assert (e.value.which, e.value.got, e.value.need) == (which, got, need)
