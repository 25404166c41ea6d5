"""Level-2 API, mirroring rblas's `level2` module (src/level2.rs) over numpy
float32 / float64 slices, computed on the GPU through librblas_b200.so:
gemv (y := alpha*op(A)*x + beta*y) and ger (A := alpha*x*y^T + A). Failures
raise (rblas panics); the slices' lengths are checked like rblas's Level-3
check_matrix, and each vector must reach its last strided element."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .level3 import _as_slice, _ptr
from .types import Layout, Transpose

__all__ = ["gemv", "ger", "gemv_dev", "ger_dev"]


def _real(y):
    dt = y.dtype if isinstance(y, np.ndarray) else None
    if dt not in (np.float32, np.float64):
        raise TypeError("real routines take float32 or float64 slices")
    return dt, "s" if dt == np.float32 else "d"


def gemv(layout, trans, m, n, alpha, a, lda, x, incx, beta, y, incy):
    """level2::gemv (src/level2.rs:11-62): y := alpha*op(A)*x + beta*y."""
    dt, p = _real(y)
    a = _as_slice(a, dt, "a")
    x = _as_slice(x, dt, "x")
    y = _as_slice(y, dt, "y", writable=True)
    err = _lib.RbError()
    st = getattr(_lib.load(), f"rb_{p}gemv")(int(Layout(layout)), int(Transpose(trans)), m, n, alpha, _ptr(a), lda,
                                             a.size, _ptr(x), incx, x.size, beta, _ptr(y), incy, y.size,
                                             C.byref(err))
    _lib.check(st, err)


def ger(layout, m, n, alpha, x, incx, y, incy, a, lda):
    """level2::ger (src/level2.rs:65-88): A := alpha*x*y^T + A."""
    dt, p = _real(a)
    x = _as_slice(x, dt, "x")
    y = _as_slice(y, dt, "y")
    a = _as_slice(a, dt, "a", writable=True)
    err = _lib.RbError()
    st = getattr(_lib.load(), f"rb_{p}ger")(int(Layout(layout)), m, n, alpha, _ptr(x), incx, x.size, _ptr(y), incy,
                                            y.size, _ptr(a), lda, a.size, C.byref(err))
    _lib.check(st, err)


def gemv_dev(layout, trans, m, n, alpha, a_ptr, lda, x_ptr, incx, beta, y_ptr, incy, dtype, stream=0):
    """Device-pointer gemv enqueued on `stream` (no synchronisation)."""
    p = "s" if np.dtype(dtype) == np.float32 else "d"
    err = _lib.RbError()
    st = getattr(_lib.load(), f"rb_{p}gemv_dev")(int(Layout(layout)), int(Transpose(trans)), m, n, alpha,
                                                 C.c_void_p(a_ptr), lda, C.c_void_p(x_ptr), incx, beta,
                                                 C.c_void_p(y_ptr), incy, C.c_void_p(stream) if stream else None,
                                                 C.byref(err))
    _lib.check(st, err)


def ger_dev(layout, m, n, alpha, x_ptr, incx, y_ptr, incy, a_ptr, lda, dtype, stream=0):
    """Device-pointer ger enqueued on `stream` (no synchronisation)."""
    p = "s" if np.dtype(dtype) == np.float32 else "d"
    err = _lib.RbError()
    st = getattr(_lib.load(), f"rb_{p}ger_dev")(int(Layout(layout)), m, n, alpha, C.c_void_p(x_ptr), incx,
                                                C.c_void_p(y_ptr), incy, C.c_void_p(a_ptr), lda,
                                                C.c_void_p(stream) if stream else None, C.byref(err))
    _lib.check(st, err)
