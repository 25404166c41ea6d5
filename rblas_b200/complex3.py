"""Complex Level-3 API, mirroring rblas's `complex3` module
(src/complex3.rs) over numpy complex64 (C32) / complex128 (C64) slices,
computed on the GPU through librblas_b200.so. Column-major, like rblas.
Failures raise (rblas panics)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .level3 import _as_slice, _ptr
from .types import Diag, Precision, Side, Transpose, Uplo

__all__ = ["gemm", "gemm_dev", "symm", "hemm", "trsm", "trmm"]


def _kind(c):
    dt = c.dtype if isinstance(c, np.ndarray) else None
    if dt == np.complex64:
        return dt, "c", _lib.RbComplex32
    if dt == np.complex128:
        return dt, "z", _lib.RbComplex64
    raise TypeError("complex routines take complex64 or complex128 slices")


def _cx(ctype, v):
    v = complex(v)
    return ctype(v.real, v.imag)


def gemm(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, prec=Precision.Plain):
    """complex3::gemm (src/complex3.rs:27-74): C := alpha*op(A)*op(B) + beta*C."""
    dt, p, ct = _kind(c)
    a = _as_slice(a, dt, "a")
    b = _as_slice(b, dt, "b")
    c = _as_slice(c, dt, "c", writable=True)
    lib = _lib.load()
    err = _lib.RbError()
    st = getattr(lib, f"rb_{p}gemm")(int(Transpose(transa)), int(Transpose(transb)), m, n, k,
                                      _cx(ct, alpha), _ptr(a), lda, a.size, _ptr(b), ldb, b.size,
                                      _cx(ct, beta), _ptr(c), ldc, c.size, int(Precision(prec)),
                                      C.byref(err))
    _lib.check(st, err)


def gemm_dev(transa, transb, m, n, k, alpha, a_ptr, lda, b_ptr, ldb, beta, c_ptr, ldc, dtype,
             prec=Precision.Plain, stream=0):
    """Device-pointer complex GEMM on `stream` (no synchronisation)."""
    p, ct = ("c", _lib.RbComplex32) if np.dtype(dtype) == np.complex64 else ("z", _lib.RbComplex64)
    lib = _lib.load()
    err = _lib.RbError()
    st = getattr(lib, f"rb_{p}gemm_dev")(int(Transpose(transa)), int(Transpose(transb)), m, n, k,
                                          _cx(ct, alpha), C.c_void_p(a_ptr), lda, C.c_void_p(b_ptr),
                                          ldb, _cx(ct, beta), C.c_void_p(c_ptr), ldc,
                                          int(Precision(prec)), C.c_void_p(stream) if stream else None,
                                          C.byref(err))
    _lib.check(st, err)


def _symm_like(name, side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc):
    dt, p, ct = _kind(c)
    a = _as_slice(a, dt, "a")
    b = _as_slice(b, dt, "b")
    c = _as_slice(c, dt, "c", writable=True)
    lib = _lib.load()
    err = _lib.RbError()
    st = getattr(lib, f"rb_{p}{name}")(int(Side(side)), int(Uplo(uplo)), m, n, _cx(ct, alpha),
                                        _ptr(a), lda, a.size, _ptr(b), ldb, b.size, _cx(ct, beta),
                                        _ptr(c), ldc, c.size, C.byref(err))
    _lib.check(st, err)


def symm(side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc):
    """complex3::symm (src/complex3.rs:130-145): A complex symmetric."""
    _symm_like("symm", side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc)


def hemm(side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc):
    """complex3::hemm (src/complex3.rs:151-166): A Hermitian."""
    _symm_like("hemm", side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc)


def trsm(side, uplo, trans, diag, m, n, alpha, a, lda, b, ldb):
    """complex3::trsm (src/complex3.rs:252-340), in place of B."""
    dt, p, ct = _kind(b)
    a = _as_slice(a, dt, "a")
    b = _as_slice(b, dt, "b", writable=True)
    lib = _lib.load()
    err = _lib.RbError()
    st = getattr(lib, f"rb_{p}trsm")(int(Side(side)), int(Uplo(uplo)), int(Transpose(trans)),
                                      int(Diag(diag)), m, n, _cx(ct, alpha), _ptr(a), lda, a.size,
                                      _ptr(b), ldb, b.size, C.byref(err))
    _lib.check(st, err)


def trmm(side, uplo, trans, diag, m, n, alpha, a, lda, b, ldb):
    """Complex triangular multiply in place of B (no rblas counterpart):
    B := alpha*op(A)*B (Left) or alpha*B*op(A) (Right); ConjTrans conjugates A."""
    dt, p, ct = _kind(b)
    a = _as_slice(a, dt, "a")
    b = _as_slice(b, dt, "b", writable=True)
    err = _lib.RbError()
    st = getattr(_lib.load(), f"rb_{p}trmm")(int(Side(side)), int(Uplo(uplo)), int(Transpose(trans)),
                                             int(Diag(diag)), m, n, _cx(ct, alpha), _ptr(a), lda, a.size, _ptr(b),
                                             ldb, b.size, C.byref(err))
    _lib.check(st, err)
