"""The oracle: TEST INFRASTRUCTURE ONLY.

ctypes bindings to ``liboracle.so`` (built from ``rblas_oracle.cpp`` by the
Makefile beside it): a CPU restatement of rblas's Level-3 GEMM path
(src/level3.rs, src/kernel/gemm.rs, src/kernel/gemm_avx2.rs, src/complex3.rs),
of its Level-1 and Level-2 routines (src/level1.rs, src/complex1.rs,
src/kernel/avx2.rs, src/level2.rs, src/complex2.rs), a compensated
double-double accuracy oracle, and numpy helpers for the normwise error
metric.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package; the product library never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

# Enum encodings shared with the product header (include/rblas_b200.h).
ROW_MAJOR, COL_MAJOR = 0, 1
NO_TRANS, TRANS, CONJ_TRANS = 0, 1, 2
UPPER, LOWER = 0, 1
LEFT, RIGHT = 0, 1
NON_UNIT, UNIT = 0, 1


class OrError(C.Structure):
    _fields_ = [("code", C.c_int32), ("which", C.c_char), ("got", C.c_uint64),
                ("min_or_need", C.c_uint64)]


def build() -> str:
    """Compile liboracle.so with the Makefile beside this file."""
    subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


_sz, _i, _f, _d = C.c_size_t, C.c_int, C.c_float, C.c_double
_pf, _pd = C.POINTER(C.c_float), C.POINTER(C.c_double)


def _declare(L):
    L.or_check_gemm.argtypes = [_i, _i, _i, _sz, _sz, _sz, _sz, _sz, _sz, _sz, _sz, _sz,
                                C.POINTER(OrError)]
    L.or_check_gemm.restype = _i
    L.or_sgemm.argtypes = [_i, _i, _i, _sz, _sz, _sz, _f, _pf, _sz, _pf, _sz, _f, _pf, _sz, _i]
    L.or_dgemm.argtypes = [_i, _i, _i, _sz, _sz, _sz, _d, _pd, _sz, _pd, _sz, _d, _pd, _sz, _i]
    L.or_ssyrk.argtypes = [_i, _i, _sz, _sz, _f, _pf, _sz, _f, _pf, _sz, _i]
    L.or_dsyrk.argtypes = [_i, _i, _sz, _sz, _d, _pd, _sz, _d, _pd, _sz, _i]
    L.or_ssymm.argtypes = [_i, _i, _sz, _sz, _f, _pf, _sz, _pf, _sz, _f, _pf, _sz, _i]
    L.or_dsymm.argtypes = [_i, _i, _sz, _sz, _d, _pd, _sz, _pd, _sz, _d, _pd, _sz, _i]
    L.or_strsm.argtypes = [_i, _i, _i, _i, _sz, _sz, _f, _pf, _sz, _pf, _sz]
    L.or_dtrsm.argtypes = [_i, _i, _i, _i, _sz, _sz, _d, _pd, _sz, _pd, _sz]
    L.or_cgemm.argtypes = [_i, _i, _sz, _sz, _sz, _f, _f, _pf, _sz, _pf, _sz, _f, _f, _pf, _sz, _i]
    L.or_zgemm.argtypes = [_i, _i, _sz, _sz, _sz, _d, _d, _pd, _sz, _pd, _sz, _d, _d, _pd, _sz, _i]
    L.or_chemm.argtypes = [_i, _i, _i, _sz, _sz, _f, _f, _pf, _sz, _pf, _sz, _f, _f, _pf, _sz, _i]
    L.or_zhemm.argtypes = [_i, _i, _i, _sz, _sz, _d, _d, _pd, _sz, _pd, _sz, _d, _d, _pd, _sz, _i]
    L.or_ctrsm.argtypes = [_i, _i, _i, _i, _sz, _sz, _f, _f, _pf, _sz, _pf, _sz]
    L.or_ztrsm.argtypes = [_i, _i, _i, _i, _sz, _sz, _d, _d, _pd, _sz, _pd, _sz]
    L.or_dd_sgemm.argtypes = [_i, _i, _i, _sz, _sz, _sz, _d, _pf, _sz, _pf, _sz, _d, _pf, _sz,
                              C.POINTER(C.c_int64), _sz, _pd, _pd, _i]
    L.or_dd_dgemm.argtypes = [_i, _i, _i, _sz, _sz, _sz, _d, _pd, _sz, _pd, _sz, _d, _pd, _sz,
                              C.POINTER(C.c_int64), _sz, _pd, _pd, _i]
    L.or_dd_core.argtypes = [_sz, _sz, _sz, _d, _pd, _pd, _d, _pd, _pd, _pd, _i]
    L.or_lcg_fill_f32.argtypes = [C.c_uint64, _i, _sz, _pf]
    L.or_lcg_fill_f32.restype = C.c_uint64
    L.or_set_force_scalar.argtypes = [_i]
    for P, t, pt in (("s", _f, _pf), ("d", _d, _pd)):
        getattr(L, f"or_{P}axpy").argtypes = [_sz, t, pt, _sz, pt, _sz]
        getattr(L, f"or_{P}dot").argtypes = [_sz, pt, _sz, pt, _sz]
        getattr(L, f"or_{P}dot").restype = t
        getattr(L, f"or_{P}scal").argtypes = [_sz, t, pt, _sz]
        getattr(L, f"or_{P}nrm2").argtypes = [_sz, pt, _sz]
        getattr(L, f"or_{P}nrm2").restype = t
        getattr(L, f"or_{P}asum").argtypes = [_sz, pt, _sz]
        getattr(L, f"or_{P}asum").restype = t
        getattr(L, f"or_{P}copy").argtypes = [_sz, pt, _sz, pt, _sz]
        getattr(L, f"or_{P}swap").argtypes = [_sz, pt, _sz, pt, _sz]
    for P, t, pt in (("c", _f, _pf), ("z", _d, _pd)):
        getattr(L, f"or_{P}axpy").argtypes = [_sz, t, t, pt, _sz, pt, _sz]
        getattr(L, f"or_{P}dot").argtypes = [_sz, pt, _sz, pt, _sz, _i, pt]
        getattr(L, f"or_{P}scal").argtypes = [_sz, t, t, pt, _sz]
        getattr(L, f"or_{P}nrm2").argtypes = [_sz, pt, _sz]
        getattr(L, f"or_{P}nrm2").restype = t
    L.or_strmm.argtypes = [_i, _i, _i, _i, _sz, _sz, _f, _pf, _sz, _pf, _sz]
    L.or_dtrmm.argtypes = [_i, _i, _i, _i, _sz, _sz, _d, _pd, _sz, _pd, _sz]
    L.or_sgemv.argtypes = [_i, _i, _sz, _sz, _f, _pf, _sz, _pf, _sz, _f, _pf, _sz]
    L.or_dgemv.argtypes = [_i, _i, _sz, _sz, _d, _pd, _sz, _pd, _sz, _d, _pd, _sz]
    L.or_sger.argtypes = [_i, _sz, _sz, _f, _pf, _sz, _pf, _sz, _pf, _sz]
    L.or_dger.argtypes = [_i, _sz, _sz, _d, _pd, _sz, _pd, _sz, _pd, _sz]
    L.or_cgemv.argtypes = [_i, _i, _sz, _sz, _f, _f, _pf, _sz, _pf, _sz, _f, _f, _pf, _sz]
    L.or_zgemv.argtypes = [_i, _i, _sz, _sz, _d, _d, _pd, _sz, _pd, _sz, _d, _d, _pd, _sz]
    L.or_cger.argtypes = [_i, _sz, _sz, _f, _f, _pf, _sz, _pf, _sz, _pf, _sz, _i]
    L.or_zger.argtypes = [_i, _sz, _sz, _d, _d, _pd, _sz, _pd, _sz, _pd, _sz, _i]
    L.or_have_avx2_fma.restype = _i


def _ptr(x: np.ndarray, ctype):
    assert x.flags["C_CONTIGUOUS"] or x.ndim == 1
    return x.ctypes.data_as(C.POINTER(ctype))


def default_threads() -> int:
    return os.cpu_count() or 1


def lcg_f32(seed: int, n: int, mode: int = 0):
    """The reference tests' LCG stream (tests/correctness.rs:21-26 mode 0,
    tests/parallel.rs:9-14 mode 1). Returns (values, final_state)."""
    out = np.empty(n, dtype=np.float32)
    s = lib().or_lcg_fill_f32(C.c_uint64(seed), mode, n, _ptr(out, C.c_float))
    return out, int(s)


def check_gemm(layout, transa, transb, m, n, k, lda, a_len, ldb, b_len, ldc, c_len):
    err = OrError()
    rc = lib().or_check_gemm(layout, transa, transb, m, n, k, lda, a_len, ldb, b_len, ldc,
                             c_len, C.byref(err))
    return rc, err


def gemm(layout, transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, threads=None):
    """rblas level3::gemm restated (src/level3.rs:32-62); writes c in place."""
    threads = default_threads() if threads is None else threads
    if c.dtype == np.float32:
        lib().or_sgemm(layout, transa, transb, m, n, k, float(alpha), _ptr(a, C.c_float), lda,
                       _ptr(b, C.c_float), ldb, float(beta), _ptr(c, C.c_float), ldc, threads)
    elif c.dtype == np.float64:
        lib().or_dgemm(layout, transa, transb, m, n, k, float(alpha), _ptr(a, C.c_double), lda,
                       _ptr(b, C.c_double), ldb, float(beta), _ptr(c, C.c_double), ldc, threads)
    elif c.dtype == np.complex64:
        lib().or_cgemm(transa, transb, m, n, k, float(np.real(alpha)), float(np.imag(alpha)),
                       _ptr(a, C.c_float), lda, _ptr(b, C.c_float), ldb, float(np.real(beta)),
                       float(np.imag(beta)), _ptr(c, C.c_float), ldc, threads)
    elif c.dtype == np.complex128:
        lib().or_zgemm(transa, transb, m, n, k, float(np.real(alpha)), float(np.imag(alpha)),
                       _ptr(a, C.c_double), lda, _ptr(b, C.c_double), ldb, float(np.real(beta)),
                       float(np.imag(beta)), _ptr(c, C.c_double), ldc, threads)
    else:
        raise TypeError(c.dtype)


def syrk(uplo, trans, n, k, alpha, a, lda, beta, c, ldc, threads=None):
    threads = default_threads() if threads is None else threads
    if c.dtype == np.float32:
        lib().or_ssyrk(uplo, trans, n, k, float(alpha), _ptr(a, C.c_float), lda, float(beta),
                       _ptr(c, C.c_float), ldc, threads)
    else:
        lib().or_dsyrk(uplo, trans, n, k, float(alpha), _ptr(a, C.c_double), lda, float(beta),
                       _ptr(c, C.c_double), ldc, threads)


def symm(side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc, threads=None, hermitian=False):
    threads = default_threads() if threads is None else threads
    if c.dtype == np.float32:
        lib().or_ssymm(side, uplo, m, n, float(alpha), _ptr(a, C.c_float), lda, _ptr(b, C.c_float),
                       ldb, float(beta), _ptr(c, C.c_float), ldc, threads)
    elif c.dtype == np.float64:
        lib().or_dsymm(side, uplo, m, n, float(alpha), _ptr(a, C.c_double), lda,
                       _ptr(b, C.c_double), ldb, float(beta), _ptr(c, C.c_double), ldc, threads)
    elif c.dtype == np.complex64:
        lib().or_chemm(int(hermitian), side, uplo, m, n, float(np.real(alpha)),
                       float(np.imag(alpha)), _ptr(a, C.c_float), lda, _ptr(b, C.c_float), ldb,
                       float(np.real(beta)), float(np.imag(beta)), _ptr(c, C.c_float), ldc, threads)
    else:
        lib().or_zhemm(int(hermitian), side, uplo, m, n, float(np.real(alpha)),
                       float(np.imag(alpha)), _ptr(a, C.c_double), lda, _ptr(b, C.c_double), ldb,
                       float(np.real(beta)), float(np.imag(beta)), _ptr(c, C.c_double), ldc,
                       threads)


def hemm(side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc, threads=None):
    symm(side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc, threads, hermitian=True)


def trsm(side, uplo, trans, diag, m, n, alpha, a, lda, b, ldb):
    if b.dtype == np.float32:
        lib().or_strsm(side, uplo, trans, diag, m, n, float(alpha), _ptr(a, C.c_float), lda,
                       _ptr(b, C.c_float), ldb)
    elif b.dtype == np.float64:
        lib().or_dtrsm(side, uplo, trans, diag, m, n, float(alpha), _ptr(a, C.c_double), lda,
                       _ptr(b, C.c_double), ldb)
    elif b.dtype == np.complex64:
        lib().or_ctrsm(side, uplo, trans, diag, m, n, float(np.real(alpha)), float(np.imag(alpha)),
                       _ptr(a, C.c_float), lda, _ptr(b, C.c_float), ldb)
    else:
        lib().or_ztrsm(side, uplo, trans, diag, m, n, float(np.real(alpha)), float(np.imag(alpha)),
                       _ptr(a, C.c_double), lda, _ptr(b, C.c_double), ldb)


def _l1(x):
    dt = np.dtype(x.dtype)
    p = {np.dtype(np.float32): "s", np.dtype(np.float64): "d", np.dtype(np.complex64): "c",
         np.dtype(np.complex128): "z"}[dt]
    ct = C.c_float if p in "sc" else C.c_double
    return p, ct


def axpy(n, alpha, x, incx, y, incy):
    """level1::axpy / complex1::axpy (src/level1.rs:17-42, src/complex1.rs:8-28), y in place."""
    p, ct = _l1(y)
    if p in "sd":
        getattr(lib(), f"or_{p}axpy")(n, float(alpha), _ptr(x, ct), incx, _ptr(y, ct), incy)
    else:
        getattr(lib(), f"or_{p}axpy")(n, float(np.real(alpha)), float(np.imag(alpha)), _ptr(x, ct), incx,
                                      _ptr(y, ct), incy)


def dot(n, x, incx, y, incy, conj=False):
    """level1::dot (src/level1.rs:45-66, contiguous through the AVX2 or scalar
    kernel of src/kernel/); complex1::dotu / dotc (src/complex1.rs:31-68)."""
    p, ct = _l1(x)
    if p in "sd":
        return float(getattr(lib(), f"or_{p}dot")(n, _ptr(x, ct), incx, _ptr(y, ct), incy))
    out = np.zeros(2, dtype=np.float32 if p == "c" else np.float64)
    getattr(lib(), f"or_{p}dot")(n, _ptr(x, ct), incx, _ptr(y, ct), incy, int(conj), _ptr(out, ct))
    return complex(out[0], out[1])


def scal(n, alpha, x, incx):
    """level1::scal / complex1::scal (src/level1.rs:70-93, src/complex1.rs:71-83), x in place."""
    p, ct = _l1(x)
    if p in "sd":
        getattr(lib(), f"or_{p}scal")(n, float(alpha), _ptr(x, ct), incx)
    else:
        getattr(lib(), f"or_{p}scal")(n, float(np.real(alpha)), float(np.imag(alpha)), _ptr(x, ct), incx)


def nrm2(n, x, incx):
    """level1::nrm2 / complex1::nrm2 (scaled sum of squares)."""
    p, ct = _l1(x)
    return float(getattr(lib(), f"or_{p}nrm2")(n, _ptr(x, ct), incx))


def asum(n, x, incx):
    """level1::asum (src/level1.rs:127-136)."""
    p, ct = _l1(x)
    return float(getattr(lib(), f"or_{p}asum")(n, _ptr(x, ct), incx))


def copy(n, x, incx, y, incy):
    """level1::copy (src/level1.rs:139-151), y in place."""
    p, ct = _l1(y)
    getattr(lib(), f"or_{p}copy")(n, _ptr(x, ct), incx, _ptr(y, ct), incy)


def swap(n, x, incx, y, incy):
    """level1::swap (src/level1.rs:155-163), x and y in place."""
    p, ct = _l1(y)
    getattr(lib(), f"or_{p}swap")(n, _ptr(x, ct), incx, _ptr(y, ct), incy)


def trmm(side, uplo, trans, diag, m, n, alpha, a, lda, b, ldb):
    """The textbook trmm (rblas has none), B in place; real types."""
    if b.dtype == np.float32:
        lib().or_strmm(side, uplo, trans, diag, m, n, float(alpha), _ptr(a, C.c_float), lda, _ptr(b, C.c_float), ldb)
    else:
        lib().or_dtrmm(side, uplo, trans, diag, m, n, float(alpha), _ptr(a, C.c_double), lda, _ptr(b, C.c_double),
                       ldb)


def gemv(layout, trans, m, n, alpha, a, lda, x, incx, beta, y, incy):
    """level2::gemv / complex2::gemv (src/level2.rs:11-62, src/complex2.rs:11-77), y in place."""
    if y.dtype == np.float32:
        lib().or_sgemv(layout, trans, m, n, float(alpha), _ptr(a, C.c_float), lda, _ptr(x, C.c_float), incx,
                       float(beta), _ptr(y, C.c_float), incy)
    elif y.dtype == np.float64:
        lib().or_dgemv(layout, trans, m, n, float(alpha), _ptr(a, C.c_double), lda, _ptr(x, C.c_double), incx,
                       float(beta), _ptr(y, C.c_double), incy)
    elif y.dtype == np.complex64:
        lib().or_cgemv(layout, trans, m, n, float(np.real(alpha)), float(np.imag(alpha)), _ptr(a, C.c_float), lda,
                       _ptr(x, C.c_float), incx, float(np.real(beta)), float(np.imag(beta)), _ptr(y, C.c_float),
                       incy)
    else:
        lib().or_zgemv(layout, trans, m, n, float(np.real(alpha)), float(np.imag(alpha)), _ptr(a, C.c_double),
                       lda, _ptr(x, C.c_double), incx, float(np.real(beta)), float(np.imag(beta)),
                       _ptr(y, C.c_double), incy)


def ger(layout, m, n, alpha, x, incx, y, incy, a, lda, conj=False):
    """level2::ger (src/level2.rs:65-88); complex: complex2::geru / gerc
    (src/complex2.rs:80-145, conj=True conjugates y). A in place."""
    if a.dtype == np.float32:
        lib().or_sger(layout, m, n, float(alpha), _ptr(x, C.c_float), incx, _ptr(y, C.c_float), incy,
                      _ptr(a, C.c_float), lda)
    elif a.dtype == np.float64:
        lib().or_dger(layout, m, n, float(alpha), _ptr(x, C.c_double), incx, _ptr(y, C.c_double), incy,
                      _ptr(a, C.c_double), lda)
    elif a.dtype == np.complex64:
        lib().or_cger(layout, m, n, float(np.real(alpha)), float(np.imag(alpha)), _ptr(x, C.c_float), incx,
                      _ptr(y, C.c_float), incy, _ptr(a, C.c_float), lda, int(conj))
    else:
        lib().or_zger(layout, m, n, float(np.real(alpha)), float(np.imag(alpha)), _ptr(x, C.c_double), incx,
                      _ptr(y, C.c_double), incy, _ptr(a, C.c_double), lda, int(conj))


def set_force_scalar(on: bool):
    lib().or_set_force_scalar(int(on))


# ---------------------------------------------------------------------------
# Double-double accuracy oracle
# ---------------------------------------------------------------------------

def dd_gemm(layout, transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c0, ldc, rows=None,
            threads=None):
    """alpha*op(A)op(B) + beta*C0 in double-double, for all rows of C or the
    given row sample. Returns (hi, lo), each len(rows) x n, row-major numpy
    arrays indexed [row_in_sample, col]."""
    threads = default_threads() if threads is None else threads
    if rows is None:
        rows_arr = None
        nrows = m
    else:
        rows_arr = np.ascontiguousarray(rows, dtype=np.int64)
        nrows = len(rows_arr)
    hi = np.empty(nrows * n, dtype=np.float64)
    lo = np.empty(nrows * n, dtype=np.float64)
    rp = rows_arr.ctypes.data_as(C.POINTER(C.c_int64)) if rows_arr is not None else None
    if a.dtype == np.float32:
        c0p = _ptr(c0, C.c_float) if (c0 is not None and beta != 0) else None
        lib().or_dd_sgemm(layout, transa, transb, m, n, k, float(alpha), _ptr(a, C.c_float), lda,
                          _ptr(b, C.c_float), ldb, float(beta), c0p, ldc, rp, nrows,
                          _ptr(hi, C.c_double), _ptr(lo, C.c_double), threads)
    else:
        c0p = _ptr(c0, C.c_double) if (c0 is not None and beta != 0) else None
        lib().or_dd_dgemm(layout, transa, transb, m, n, k, float(alpha), _ptr(a, C.c_double), lda,
                          _ptr(b, C.c_double), ldb, float(beta), c0p, ldc, rp, nrows,
                          _ptr(hi, C.c_double), _ptr(lo, C.c_double), threads)
    # col-major nrows x n -> [row, col]
    return hi.reshape(n, nrows).T.copy(), lo.reshape(n, nrows).T.copy()


def dd_core(am, bm, alpha=1.0, beta=0.0, c0=None, threads=None):
    """Double-double alpha*am@bm + beta*c0 for float64 2-D numpy arrays."""
    threads = default_threads() if threads is None else threads
    nrows, k = am.shape
    k2, n = bm.shape
    assert k == k2
    amc = np.asfortranarray(am, dtype=np.float64)
    bmc = np.asfortranarray(bm, dtype=np.float64)
    c0c = np.asfortranarray(c0, dtype=np.float64) if c0 is not None else None
    hi = np.empty(nrows * n, dtype=np.float64)
    lo = np.empty(nrows * n, dtype=np.float64)
    L = lib()
    L.or_dd_core(nrows, n, k, float(alpha), amc.ctypes.data_as(_pd), bmc.ctypes.data_as(_pd),
                 float(beta), c0c.ctypes.data_as(_pd) if c0c is not None else None,
                 hi.ctypes.data_as(_pd), lo.ctypes.data_as(_pd), threads)
    return hi.reshape(n, nrows).T.copy(), lo.reshape(n, nrows).T.copy()


def dd_complex_gemm(opa, opb, alpha, beta, c0=None, threads=None):
    """Double-double oracle for complex alpha*opa@opb + beta*c0 (2-D complex
    numpy arrays, op() already applied). Returns (hi, lo) complex arrays."""
    ar, ai = opa.real.astype(np.float64), opa.imag.astype(np.float64)
    br, bi = opb.real.astype(np.float64), opb.imag.astype(np.float64)
    # [Pr; Pi] = [[Ar, -Ai], [Ai, Ar]] @ [Br; Bi], exact block form
    top = np.hstack([ar, -ai])
    bot = np.hstack([ai, ar])
    bb = np.vstack([br, bi])
    prh, prl = dd_core(top, bb, threads=threads)
    pih, pil = dd_core(bot, bb, threads=threads)
    p = (prh + prl) + 1j * (pih + pil)
    res = alpha * p
    if c0 is not None and beta != 0:
        res = res + beta * c0.astype(np.complex128)
    return res, np.zeros_like(res)


def stored_2d(x, rows, cols, ld, layout):
    """View a flat BLAS buffer as its stored rows x cols matrix."""
    if layout == COL_MAJOR:
        return np.lib.stride_tricks.as_strided(
            x, shape=(rows, cols), strides=(x.itemsize, x.itemsize * ld))
    return np.lib.stride_tricks.as_strided(
        x, shape=(rows, cols), strides=(x.itemsize * ld, x.itemsize))


def normwise_error(c, hi, lo, alpha, a_norm_f, b_norm_f, beta, c0_norm_f):
    """||C - C_ref||_F / (|alpha| ||A||_F ||B||_F + |beta| ||C0||_F) with
    C_ref = hi + lo from the double-double oracle (all 2-D, same shape)."""
    diff = (c.astype(np.float64) - hi) - lo
    num = np.sqrt(np.sum(diff * diff))
    den = abs(alpha) * a_norm_f * b_norm_f + abs(beta) * c0_norm_f
    return float(num / den) if den > 0 else float(num)


def unit_roundoff(dtype) -> float:
    return {np.float32: 2.0 ** -24, np.float64: 2.0 ** -53}[np.dtype(dtype).type]
