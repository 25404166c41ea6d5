"""Complex Level-2 API, mirroring rblas's `complex2` module
(src/complex2.rs) over numpy complex64 / complex128 slices, computed on the
GPU through librblas_b200.so: gemv (op = none, transpose or conjugate
transpose), geru (A := alpha*x*y^T + A) and gerc (A := alpha*x*y^H + A)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .complex3 import _cx, _kind
from .level3 import _as_slice, _ptr
from .types import Layout, Transpose

__all__ = ["gemv", "geru", "gerc", "gemv_dev", "geru_dev", "gerc_dev"]


def gemv(layout, trans, m, n, alpha, a, lda, x, incx, beta, y, incy):
    """complex2::gemv (src/complex2.rs:11-77): y := alpha*op(A)*x + beta*y."""
    dt, p, ct = _kind(y)
    a = _as_slice(a, dt, "a")
    x = _as_slice(x, dt, "x")
    y = _as_slice(y, dt, "y", writable=True)
    err = _lib.RbError()
    st = getattr(_lib.load(), f"rb_{p}gemv")(int(Layout(layout)), int(Transpose(trans)), m, n, _cx(ct, alpha),
                                             _ptr(a), lda, a.size, _ptr(x), incx, x.size, _cx(ct, beta), _ptr(y),
                                             incy, y.size, C.byref(err))
    _lib.check(st, err)


def _rank1(name, layout, m, n, alpha, x, incx, y, incy, a, lda):
    dt, p, ct = _kind(a)
    x = _as_slice(x, dt, "x")
    y = _as_slice(y, dt, "y")
    a = _as_slice(a, dt, "a", writable=True)
    err = _lib.RbError()
    st = getattr(_lib.load(), f"rb_{p}{name}")(int(Layout(layout)), m, n, _cx(ct, alpha), _ptr(x), incx, x.size,
                                               _ptr(y), incy, y.size, _ptr(a), lda, a.size, C.byref(err))
    _lib.check(st, err)


def geru(layout, m, n, alpha, x, incx, y, incy, a, lda):
    """complex2::geru (src/complex2.rs:80-94): A := alpha*x*y^T + A."""
    _rank1("geru", layout, m, n, alpha, x, incx, y, incy, a, lda)


def gerc(layout, m, n, alpha, x, incx, y, incy, a, lda):
    """complex2::gerc (src/complex2.rs:97-111): A := alpha*x*y^H + A."""
    _rank1("gerc", layout, m, n, alpha, x, incx, y, incy, a, lda)


def gemv_dev(layout, trans, m, n, alpha, a_ptr, lda, x_ptr, incx, beta, y_ptr, incy, dtype, stream=0):
    p, ct = ("c", _lib.RbComplex32) if np.dtype(dtype) == np.complex64 else ("z", _lib.RbComplex64)
    err = _lib.RbError()
    st = getattr(_lib.load(), f"rb_{p}gemv_dev")(int(Layout(layout)), int(Transpose(trans)), m, n, _cx(ct, alpha),
                                                 C.c_void_p(a_ptr), lda, C.c_void_p(x_ptr), incx, _cx(ct, beta),
                                                 C.c_void_p(y_ptr), incy, C.c_void_p(stream) if stream else None,
                                                 C.byref(err))
    _lib.check(st, err)


def _rank1_dev(name, layout, m, n, alpha, x_ptr, incx, y_ptr, incy, a_ptr, lda, dtype, stream):
    p, ct = ("c", _lib.RbComplex32) if np.dtype(dtype) == np.complex64 else ("z", _lib.RbComplex64)
    err = _lib.RbError()
    st = getattr(_lib.load(), f"rb_{p}{name}_dev")(int(Layout(layout)), m, n, _cx(ct, alpha), C.c_void_p(x_ptr),
                                                   incx, C.c_void_p(y_ptr), incy, C.c_void_p(a_ptr), lda,
                                                   C.c_void_p(stream) if stream else None, C.byref(err))
    _lib.check(st, err)


def geru_dev(layout, m, n, alpha, x_ptr, incx, y_ptr, incy, a_ptr, lda, dtype, stream=0):
    _rank1_dev("geru", layout, m, n, alpha, x_ptr, incx, y_ptr, incy, a_ptr, lda, dtype, stream)


def gerc_dev(layout, m, n, alpha, x_ptr, incx, y_ptr, incy, a_ptr, lda, dtype, stream=0):
    _rank1_dev("gerc", layout, m, n, alpha, x_ptr, incx, y_ptr, incy, a_ptr, lda, dtype, stream)
