"""Complex Level-1 API, mirroring rblas's `complex1` module (src/complex1.rs)
over numpy complex64 / complex128 slices, computed on the GPU through
librblas_b200.so: axpy, dotu, dotc, scal, nrm2. axpy and scal give rblas's
elements exactly (its complex multiply, src/complex.rs:101-111); dotu, dotc
and nrm2 sum in a fixed parallel order and agree with rblas's loop within
rounding."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .complex3 import _cx, _kind
from .level1 import _call, _st
from .level3 import _as_slice, _ptr

__all__ = ["axpy", "dotu", "dotc", "scal", "nrm2", "axpy_dev", "dotu_dev", "dotc_dev", "scal_dev", "nrm2_dev"]


def axpy(n, alpha, x, incx, y, incy):
    """complex1::axpy (src/complex1.rs:8-27): y := alpha*x + y."""
    dt, p, ct = _kind(y)
    x = _as_slice(x, dt, "x")
    y = _as_slice(y, dt, "y", writable=True)
    _call(f"rb_{p}axpy", n, _cx(ct, alpha), _ptr(x), incx, x.size, _ptr(y), incy, y.size)


def _dot(name, n, x, incx, y, incy):
    dt, p, ct = _kind(x)
    x = _as_slice(x, dt, "x")
    y = _as_slice(y, dt, "y")
    out = ct()
    _call(f"rb_{p}{name}", n, _ptr(x), incx, x.size, _ptr(y), incy, y.size, C.byref(out))
    return complex(out.re, out.im)


def dotu(n, x, incx, y, incy):
    """complex1::dotu (src/complex1.rs:31-47): sum x_i * y_i."""
    return _dot("dotu", n, x, incx, y, incy)


def dotc(n, x, incx, y, incy):
    """complex1::dotc (src/complex1.rs:51-67): sum conj(x_i) * y_i."""
    return _dot("dotc", n, x, incx, y, incy)


def scal(n, alpha, x, incx):
    """complex1::scal (src/complex1.rs:71-81): x := alpha*x."""
    dt, p, ct = _kind(x)
    x = _as_slice(x, dt, "x", writable=True)
    _call(f"rb_{p}scal", n, _cx(ct, alpha), _ptr(x), incx, x.size)


def nrm2(n, x, incx):
    """complex1::nrm2 (src/complex1.rs:86-112): ||x||_2 over the components re, im."""
    dt, p, ct = _kind(x)
    x = _as_slice(x, dt, "x")
    out = (C.c_float if p == "c" else C.c_double)()
    _call(f"rb_{'sc' if p == 'c' else 'dz'}nrm2", n, _ptr(x), incx, x.size, C.byref(out))
    return out.value


# ---- device pointers (enqueued on `stream`, no synchronisation) ----------------

def _pc(dtype):
    return ("c", _lib.RbComplex32) if np.dtype(dtype) == np.complex64 else ("z", _lib.RbComplex64)


def axpy_dev(n, alpha, x_ptr, incx, y_ptr, incy, dtype, stream=0):
    p, ct = _pc(dtype)
    _call(f"rb_{p}axpy_dev", n, _cx(ct, alpha), C.c_void_p(x_ptr), incx, C.c_void_p(y_ptr), incy, _st(stream))


def scal_dev(n, alpha, x_ptr, incx, dtype, stream=0):
    p, ct = _pc(dtype)
    _call(f"rb_{p}scal_dev", n, _cx(ct, alpha), C.c_void_p(x_ptr), incx, _st(stream))


def dotu_dev(n, x_ptr, incx, y_ptr, incy, result_ptr, dtype, stream=0):
    p, _ = _pc(dtype)
    _call(f"rb_{p}dotu_dev", n, C.c_void_p(x_ptr), incx, C.c_void_p(y_ptr), incy, C.c_void_p(result_ptr),
          _st(stream))


def dotc_dev(n, x_ptr, incx, y_ptr, incy, result_ptr, dtype, stream=0):
    p, _ = _pc(dtype)
    _call(f"rb_{p}dotc_dev", n, C.c_void_p(x_ptr), incx, C.c_void_p(y_ptr), incy, C.c_void_p(result_ptr),
          _st(stream))


def nrm2_dev(n, x_ptr, incx, result_ptr, dtype, stream=0):
    p, _ = _pc(dtype)
    _call(f"rb_{'sc' if p == 'c' else 'dz'}nrm2_dev", n, C.c_void_p(x_ptr), incx, C.c_void_p(result_ptr),
          _st(stream))
