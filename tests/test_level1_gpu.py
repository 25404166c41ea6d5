"""Level 1 on the GPU through the C ABI, against the oracle.

axpy, scal, copy and swap must equal the oracle bit for bit (they compute
each element as rblas does). dot / dotu / dotc / asum / nrm2 sum in a fixed
parallel order, so they are checked three ways: (1) on integer-valued data
whose every partial sum is exact, they equal the exact sum bit for bit, which
catches a dropped or doubled element at any size; (2) on random data, their
error against an exactly summed reference stays within the fixed-order bound
(chain + tree length) x eps x sum|terms|, written below as `_tol`; (3) two
calls give the same bits. Sizes cover the 16-byte vector path with and
without its unrolled loop, ragged tails, strides, zero strides and
misaligned device pointers.
"""
from __future__ import annotations

import math
import zlib

import numpy as np
import pytest

import oracle
import rblas_b200 as rb
from rblas_b200 import complex1, level1

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

NTH = 148 * 4 * 256  # threads of a Level-1 grid
SIZES = [1, 3, 17, 1000, 100_003, 2_500_007]


def _rng(*k):
    return np.random.default_rng(zlib.crc32(repr(k).encode()))


def _vec(rng, n, dt):
    if np.issubdtype(dt, np.complexfloating):
        return (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(dt)
    return rng.standard_normal(n).astype(dt)


def _two_prod(a, b):
    """Exact a*b = p + e for float64 arrays (Veltkamp split, Dekker product)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)

    def split(v):
        c = 134217729.0 * v
        hi = c - (c - v)
        return hi, v - hi

    p = a * b
    ah, al = split(a)
    bh, bl = split(b)
    e = ((ah * bh - p) + ah * bl + al * bh) + al * bl
    return p, e


def _exact_sum_of_products(pairs):
    parts = []
    for a, b, sgn in pairs:
        p, e = _two_prod(a, b)
        parts.append(sgn * p)
        parts.append(sgn * e)
    return math.fsum(np.concatenate(parts).tolist())


def _eps(dt):
    return float(np.finfo(np.float32 if dt in (np.float32, np.complex64) else np.float64).eps)


def _tol(n, dt, scale):
    """Fixed-order bound: a thread folds at most ceil(n/NTH) 16-byte vectors
    of up to 4 scalars, then a 256-way tree and a 592-way fold."""
    chain = 4 * (-(-n // NTH)) + 4 + 8 + 3 + 8
    return (chain + 8) * _eps(dt) * scale


# ---- elementwise: bit-identical to the oracle ---------------------------------

@pytest.mark.parametrize("dt", [np.float32, np.float64, np.complex64, np.complex128])
@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("incx,incy", [(1, 1), (2, 3)])
def test_axpy_scal_copy_swap_exact(dt, n, incx, incy):
    cx = np.issubdtype(dt, np.complexfloating)
    if n > 100_003 and (incx, incy) != (1, 1):
        pytest.skip("large strided sizes add nothing over 100003")
    rng = _rng("ew", np.dtype(dt).name, n, incx)
    x = _vec(rng, (n - 1) * incx + 1, dt)
    y0 = _vec(rng, (n - 1) * incy + 1, dt)
    alpha = (0.75 - 1.25j) if cx else 0.75
    mod = complex1 if cx else level1

    y, want = y0.copy(), y0.copy()
    mod.axpy(n, alpha, x, incx, y, incy)
    oracle.axpy(n, alpha, x, incx, want, incy)
    assert np.array_equal(y.view(np.uint8), want.view(np.uint8))

    s, want = x.copy(), x.copy()
    mod.scal(n, alpha, s, incx)
    oracle.scal(n, alpha, want, incx)
    assert np.array_equal(s.view(np.uint8), want.view(np.uint8))

    if not cx:  # rblas's copy / swap are real (level1::copy / swap)
        y, want = y0.copy(), y0.copy()
        level1.copy(n, x, incx, y, incy)
        oracle.copy(n, x, incx, want, incy)
        assert np.array_equal(y, want)
        a, b, wa, wb = x.copy(), y0.copy(), x.copy(), y0.copy()
        level1.swap(n, a, incx, b, incy)
        oracle.swap(n, wa, incx, wb, incy)
        assert np.array_equal(a, wa) and np.array_equal(b, wb)


def test_scal_special_values_follow_rblas():
    x = np.array([np.inf, np.nan, -0.0, 1.0, -3.0])
    want = x.copy()
    oracle.scal(5, 0.0, want, 1)
    level1.scal(5, 0.0, x, 1)  # 0*inf = nan, 0*(-0) = -0: a multiply, not a fill
    assert np.isnan(x[:2]).all() and np.isnan(want[:2]).all()  # NaN payloads differ by vendor
    assert np.array_equal(x[2:].view(np.uint64), want[2:].view(np.uint64))


def test_copy_with_zero_strides():
    x = np.arange(1.0, 8.0)
    y = np.zeros(1)
    level1.copy(7, x, 1, y, 0)  # the last element stays, as in rblas's loop
    assert y[0] == 7.0
    y = np.zeros(4)
    level1.copy(4, x, 0, y, 1)  # broadcast x[0]
    assert list(y) == [1.0] * 4


# ---- reductions: exact on integer data -----------------------------------------

@pytest.mark.parametrize("dt", [np.float32, np.float64, np.complex64, np.complex128])
@pytest.mark.parametrize("n", SIZES + [5_000_011])
def test_reductions_exact_on_integer_data(dt, n):
    """Entries in {-1, 0, 1}: every partial sum is an integer below 2^24, so
    any order of summation gives the exact value; a lost or doubled element
    changes it."""
    cx = np.issubdtype(dt, np.complexfloating)
    rng = _rng("int", np.dtype(dt).name, n)
    ints = lambda: rng.integers(-1, 2, n).astype(np.float64)
    if cx:
        x = (ints() + 1j * ints()).astype(dt)
        y = (ints() + 1j * ints()).astype(dt)
        xd, yd = x.astype(np.complex128), y.astype(np.complex128)
        assert complex1.dotu(n, x, 1, y, 1) == complex(np.sum(xd * yd))
        assert complex1.dotc(n, x, 1, y, 1) == complex(np.sum(np.conj(xd) * yd))
    else:
        x, y = ints().astype(dt), ints().astype(dt)
        assert level1.dot(n, x, 1, y, 1) == float(np.dot(x.astype(np.float64), y))
        assert level1.asum(n, x, 1) == float(np.sum(np.abs(x.astype(np.float64))))


@pytest.mark.parametrize("dt", [np.float32, np.float64, np.complex64, np.complex128])
@pytest.mark.parametrize("n,incx", [(1000, 1), (100_003, 1), (2_500_007, 1), (100_003, 3)])
def test_nrm2_finds_planted_elements(dt, n, incx):
    """x = 0 except a 3 and a 4 at positions spread over the vector (head,
    vector boundaries, the unrolled loop, the ragged tail): the scaled sum of
    squares gives exactly 5 in any merge order."""
    cx = np.issubdtype(dt, np.complexfloating)
    lenx = (n - 1) * incx + 1
    for j, k in [(0, n - 1), (n - 1, 0), (n // 2, n // 2 + 1), (NTH * 4 % n, n - 2), (7, NTH % n)]:
        if j == k:
            continue
        x = np.zeros(lenx, dt)
        x[j * incx] = 3.0
        x[k * incx] = (4j if cx else 4.0)
        got = complex1.nrm2(n, x, incx) if cx else level1.nrm2(n, x, incx)
        assert got == 5.0, (j, k, got)


# ---- reductions: random data within the fixed-order bound -----------------------

@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("incx,incy", [(1, 1), (2, 3)])
def test_real_reductions_within_bound(dt, n, incx, incy):
    if n > 100_003 and (incx, incy) != (1, 1):
        pytest.skip("large strided sizes add nothing over 100003")
    rng = _rng("red", np.dtype(dt).name, n, incx)
    x = _vec(rng, (n - 1) * incx + 1, dt)
    y = _vec(rng, (n - 1) * incy + 1, dt)
    xs, ys = x[::incx][:n].astype(np.float64), y[::incy][:n].astype(np.float64)

    exact = _exact_sum_of_products([(xs, ys, 1.0)])
    got = level1.dot(n, x, incx, y, incy)
    assert abs(got - exact) <= _tol(n, dt, float(np.sum(np.abs(xs * ys)))), (got, exact)
    ref = oracle.dot(n, x, incx, y, incy)  # rblas's own order, for the record of agreement
    assert abs(got - ref) <= _tol(n, dt, float(np.sum(np.abs(xs * ys)))) + n * _eps(dt) * float(np.sum(np.abs(xs * ys)))

    exact = math.fsum(np.abs(xs).tolist())
    assert abs(level1.asum(n, x, incx) - exact) <= _tol(n, dt, exact)

    ss = _exact_sum_of_products([(xs, xs, 1.0)])
    want = math.sqrt(ss)
    got = level1.nrm2(n, x, incx)
    assert abs(got - want) <= 4 * _tol(n, dt, want), (got, want)
    assert abs(got - oracle.nrm2(n, x, incx)) <= 4 * _tol(n, dt, want) + 4 * n * _eps(dt) * want


@pytest.mark.parametrize("dt", [np.complex64, np.complex128])
@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("incx,incy", [(1, 1), (2, 1)])
def test_complex_reductions_within_bound(dt, n, incx, incy):
    if n > 100_003 and (incx, incy) != (1, 1):
        pytest.skip("large strided sizes add nothing over 100003")
    rng = _rng("cred", np.dtype(dt).name, n, incx)
    x = _vec(rng, (n - 1) * incx + 1, dt)
    y = _vec(rng, (n - 1) * incy + 1, dt)
    xs, ys = x[::incx][:n].astype(np.complex128), y[::incy][:n].astype(np.complex128)
    xr, xi, yr, yi = xs.real, xs.imag, ys.real, ys.imag
    scale = float(np.sum((np.abs(xr) + np.abs(xi)) * (np.abs(yr) + np.abs(yi))))
    for conj, fn in ((False, complex1.dotu), (True, complex1.dotc)):
        s = -1.0 if conj else 1.0
        re = _exact_sum_of_products([(xr, yr, 1.0), (xi, yi, -s)])
        im = _exact_sum_of_products([(xr, yi, 1.0), (xi, yr, s)])
        got = fn(n, x, incx, y, incy)
        assert abs(got.real - re) <= _tol(n, dt, scale) and abs(got.imag - im) <= _tol(n, dt, scale), (got, re, im)
    want = math.sqrt(_exact_sum_of_products([(xr, xr, 1.0), (xi, xi, 1.0)]))
    assert abs(complex1.nrm2(n, x, incx) - want) <= 4 * _tol(2 * n, dt, want)


def test_reductions_are_deterministic():
    rng = _rng("det")
    x = rng.standard_normal(3_000_001).astype(np.float32)
    y = rng.standard_normal(3_000_001).astype(np.float32)
    a = [level1.dot(x.size, x, 1, y, 1) for _ in range(3)]
    b = [level1.nrm2(x.size, x, 1) for _ in range(3)]
    assert len({np.float32(v).tobytes() for v in a}) == 1
    assert len({np.float32(v).tobytes() for v in b}) == 1


def test_nrm2_overflow_underflow_and_special_values():
    for dt, big, tiny in ((np.float64, 1e200, 1e-200), (np.float32, 1e30, 1e-30)):
        n = 100_003
        got = level1.nrm2(n, np.full(n, big, dt), 1)
        assert math.isfinite(got) and abs(got / (float(dt(big)) * math.sqrt(n)) - 1) < 1e-4
        got = level1.nrm2(n, np.full(n, tiny, dt), 1)
        assert got > 0 and abs(got / (float(dt(tiny)) * math.sqrt(n)) - 1) < 1e-4
    x = np.ones(100_003)
    x[77_777] = np.inf
    assert math.isinf(level1.nrm2(x.size, x, 1)) and math.isinf(oracle.nrm2(x.size, x, 1))
    x[50_000] = np.nan
    assert math.isnan(level1.nrm2(x.size, x, 1)) and math.isnan(oracle.nrm2(x.size, x, 1))
    z = np.zeros(1000)
    z[999] = np.nan  # a NaN in a partial that saw no nonzero element
    assert math.isnan(level1.nrm2(z.size, z, 1))
    assert level1.nrm2(1000, np.zeros(1000), 1) == 0.0


def test_zero_strides_in_reductions():
    x = np.array([2.0, 5.0, 7.0])
    y = np.arange(1.0, 11.0)
    assert level1.asum(10, x, 0) == 20.0
    assert complex1.dotu(4, np.array([1 + 1j]), 0, np.array([1j, 2, 3, 4j]), 1) == (1 + 1j) * (5 + 5j)
    with pytest.raises(rb.ZeroStride):  # rblas asserts positive strides off the contiguous path
        level1.dot(1, x, 0, y, 0)


def test_strided_gaps_come_back_unchanged():
    y = np.arange(10.0)
    level1.axpy(4, 1.0, np.ones(4), 1, y, 3)  # touches 0, 3, 6, 9
    assert list(y) == [1.0, 1.0, 2.0, 4.0, 4.0, 5.0, 7.0, 7.0, 8.0, 10.0]
    x = np.arange(7.0)
    level1.scal(3, -1.0, x, 3)
    assert list(x) == [-0.0, 1.0, 2.0, -3.0, 4.0, 5.0, -6.0]


def test_launches_native_kernels():
    before = rb.launch_count()
    level1.dot(1000, np.ones(1000), 1, np.ones(1000), 1)
    level1.axpy(1000, 2.0, np.ones(1000), 1, np.ones(1000), 1)
    assert rb.launch_count() - before == 3  # partial + final reduction, one elementwise kernel


# ---- device pointers ------------------------------------------------------------

@pytest.mark.parametrize("dt", [torch.float32, torch.float64])
@pytest.mark.parametrize("offset", [0, 1])
def test_device_pointer_forms(dt, offset):
    """The _dev entry points on torch memory, 16-byte aligned or not (offset
    1 element: the one-element-per-step path), against the host forms."""
    n = 1_000_003
    npdt = np.float32 if dt == torch.float32 else np.float64
    g = torch.Generator(device="cuda").manual_seed(5)
    xb = torch.randn(n + 1, device="cuda", dtype=dt, generator=g)
    yb = torch.randn(n + 1, device="cuda", dtype=dt, generator=g)
    x, y = xb[offset:offset + n], yb[offset:offset + n]
    xh, yh = x.cpu().numpy(), y.cpu().numpy()
    out = torch.zeros(4, device="cuda", dtype=dt)
    level1.dot_dev(n, x.data_ptr(), 1, y.data_ptr(), 1, out.data_ptr(), npdt)
    level1.asum_dev(n, x.data_ptr(), 1, out[1:].data_ptr(), npdt)
    level1.nrm2_dev(n, x.data_ptr(), 1, out[2:].data_ptr(), npdt)
    torch.cuda.synchronize()
    r = out.cpu().numpy()
    xs = xh.astype(np.float64)
    assert abs(r[0] - _exact_sum_of_products([(xs, yh, 1.0)])) <= _tol(n, npdt, float(np.sum(np.abs(xs * yh))))
    assert abs(r[1] - math.fsum(np.abs(xs).tolist())) <= _tol(n, npdt, float(np.sum(np.abs(xs))))
    want = math.sqrt(_exact_sum_of_products([(xs, xs, 1.0)]))
    assert abs(r[2] - want) <= 4 * _tol(n, npdt, want)
    if offset == 0:  # same alignment as the host path's staging buffer: the same bits
        assert r[0] == npdt(level1.dot(n, xh, 1, yh, 1))
    want_y = yh.copy()
    oracle.axpy(n, 1.5, xh, 1, want_y, 1)
    level1.axpy_dev(n, 1.5, x.data_ptr(), 1, y.data_ptr(), 1, npdt)
    torch.cuda.synchronize()
    assert np.array_equal(y.cpu().numpy(), want_y)
    level1.swap_dev(n, x.data_ptr(), 1, y.data_ptr(), 1, npdt)
    level1.scal_dev(n, -2.0, x.data_ptr(), 1, npdt)
    level1.copy_dev(n, x.data_ptr(), 1, y.data_ptr(), 1, npdt)
    torch.cuda.synchronize()
    want_x = want_y.copy()
    oracle.scal(n, -2.0, want_x, 1)
    assert np.array_equal(x.cpu().numpy(), want_x) and np.array_equal(y.cpu().numpy(), want_x)


def test_complex_device_pointer_forms():
    n = 300_001
    g = torch.Generator(device="cuda").manual_seed(9)
    x = torch.randn(n, device="cuda", dtype=torch.complex64, generator=g)
    y = torch.randn(n, device="cuda", dtype=torch.complex64, generator=g)
    xh, yh = x.cpu().numpy(), y.cpu().numpy()
    out = torch.zeros(2, device="cuda", dtype=torch.complex64)
    complex1.dotc_dev(n, x.data_ptr(), 1, y.data_ptr(), 1, out.data_ptr(), np.complex64)
    torch.cuda.synchronize()
    assert out[0].item() == np.complex64(complex1.dotc(n, xh, 1, yh, 1))
    want = yh.copy()
    oracle.axpy(n, 0.5 + 2j, xh, 1, want, 1)
    complex1.axpy_dev(n, 0.5 + 2j, x.data_ptr(), 1, y.data_ptr(), 1, np.complex64)
    torch.cuda.synchronize()
    assert np.array_equal(y.cpu().numpy().view(np.uint8), want.view(np.uint8))
    r = torch.zeros(1, device="cuda", dtype=torch.float32)
    complex1.nrm2_dev(n, x.data_ptr(), 1, r.data_ptr(), np.complex64)
    torch.cuda.synchronize()
    assert r.item() == np.float32(complex1.nrm2(n, xh, 1))
