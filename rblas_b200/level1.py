"""Level-1 API, mirroring rblas's `level1` module (src/level1.rs) over numpy
float32 / float64 slices, computed on the GPU through librblas_b200.so:
axpy, dot, scal, nrm2, asum, copy, swap. Vectors are strided (incx, incy);
failures raise where rblas panics (a zero stride where it asserts a positive
one: ZeroStride; a slice shorter than its last strided element:
BufferTooSmall). axpy / scal / copy / swap give rblas's elements exactly;
the reductions sum in a fixed parallel order (the same result on every call)
and agree with rblas's sequential loop within rounding."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .level2 import _real
from .level3 import _as_slice, _ptr

__all__ = ["axpy", "dot", "scal", "nrm2", "asum", "copy", "swap",
           "axpy_dev", "dot_dev", "scal_dev", "nrm2_dev", "asum_dev", "copy_dev", "swap_dev"]


def _ctype(p):
    return C.c_float if p == "s" else C.c_double


def _call(name, *args):
    err = _lib.RbError()
    st = getattr(_lib.load(), name)(*args, C.byref(err))
    _lib.check(st, err)


def axpy(n, alpha, x, incx, y, incy):
    """level1::axpy (src/level1.rs:17-41): y := alpha*x + y, each element fma(alpha, x_i, y_i)."""
    dt, p = _real(y)
    x = _as_slice(x, dt, "x")
    y = _as_slice(y, dt, "y", writable=True)
    _call(f"rb_{p}axpy", n, alpha, _ptr(x), incx, x.size, _ptr(y), incy, y.size)


def dot(n, x, incx, y, incy):
    """level1::dot (src/level1.rs:45-66): x^T y."""
    dt, p = _real(x)
    x = _as_slice(x, dt, "x")
    y = _as_slice(y, dt, "y")
    out = _ctype(p)()
    _call(f"rb_{p}dot", n, _ptr(x), incx, x.size, _ptr(y), incy, y.size, C.byref(out))
    return out.value


def scal(n, alpha, x, incx):
    """level1::scal (src/level1.rs:70-86): x := alpha*x."""
    dt, p = _real(x)
    x = _as_slice(x, dt, "x", writable=True)
    _call(f"rb_{p}scal", n, alpha, _ptr(x), incx, x.size)


def nrm2(n, x, incx):
    """level1::nrm2 (src/level1.rs:96-123): ||x||_2 by the scaled sum of squares."""
    dt, p = _real(x)
    x = _as_slice(x, dt, "x")
    out = _ctype(p)()
    _call(f"rb_{p}nrm2", n, _ptr(x), incx, x.size, C.byref(out))
    return out.value


def asum(n, x, incx):
    """level1::asum (src/level1.rs:127-135): sum of |x_i|."""
    dt, p = _real(x)
    x = _as_slice(x, dt, "x")
    out = _ctype(p)()
    _call(f"rb_{p}asum", n, _ptr(x), incx, x.size, C.byref(out))
    return out.value


def copy(n, x, incx, y, incy):
    """level1::copy (src/level1.rs:139-151): y := x."""
    dt, p = _real(y)
    x = _as_slice(x, dt, "x")
    y = _as_slice(y, dt, "y", writable=True)
    _call(f"rb_{p}copy", n, _ptr(x), incx, x.size, _ptr(y), incy, y.size)


def swap(n, x, incx, y, incy):
    """level1::swap (src/level1.rs:155-163): x <-> y."""
    dt, p = _real(y)
    x = _as_slice(x, dt, "x", writable=True)
    y = _as_slice(y, dt, "y", writable=True)
    _call(f"rb_{p}swap", n, _ptr(x), incx, x.size, _ptr(y), incy, y.size)


# ---- device pointers (enqueued on `stream`, no synchronisation) ----------------

def _p(dtype):
    return "s" if np.dtype(dtype) == np.float32 else "d"


def _st(stream):
    return C.c_void_p(stream) if stream else None


def axpy_dev(n, alpha, x_ptr, incx, y_ptr, incy, dtype, stream=0):
    _call(f"rb_{_p(dtype)}axpy_dev", n, alpha, C.c_void_p(x_ptr), incx, C.c_void_p(y_ptr), incy, _st(stream))


def scal_dev(n, alpha, x_ptr, incx, dtype, stream=0):
    _call(f"rb_{_p(dtype)}scal_dev", n, alpha, C.c_void_p(x_ptr), incx, _st(stream))


def copy_dev(n, x_ptr, incx, y_ptr, incy, dtype, stream=0):
    _call(f"rb_{_p(dtype)}copy_dev", n, C.c_void_p(x_ptr), incx, C.c_void_p(y_ptr), incy, _st(stream))


def swap_dev(n, x_ptr, incx, y_ptr, incy, dtype, stream=0):
    _call(f"rb_{_p(dtype)}swap_dev", n, C.c_void_p(x_ptr), incx, C.c_void_p(y_ptr), incy, _st(stream))


def dot_dev(n, x_ptr, incx, y_ptr, incy, result_ptr, dtype, stream=0):
    """x^T y written to device memory at result_ptr."""
    _call(f"rb_{_p(dtype)}dot_dev", n, C.c_void_p(x_ptr), incx, C.c_void_p(y_ptr), incy, C.c_void_p(result_ptr),
          _st(stream))


def asum_dev(n, x_ptr, incx, result_ptr, dtype, stream=0):
    _call(f"rb_{_p(dtype)}asum_dev", n, C.c_void_p(x_ptr), incx, C.c_void_p(result_ptr), _st(stream))


def nrm2_dev(n, x_ptr, incx, result_ptr, dtype, stream=0):
    _call(f"rb_{_p(dtype)}nrm2_dev", n, C.c_void_p(x_ptr), incx, C.c_void_p(result_ptr), _st(stream))
