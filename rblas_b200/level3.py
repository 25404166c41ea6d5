"""Real Level-3 API, mirroring rblas's `level3` module (src/level3.rs) over
numpy host slices, computed on the GPU through librblas_b200.so.

Arguments follow the Rust signatures one for one (slices are 1-D numpy
arrays whose length is the slice length). As in rblas, `gemm` fails loudly
(raises) on a precondition violation and `try_gemm` returns the error
(None on success). `prec` selects the arithmetic form; the default is the
plain form, the drop-in.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .types import Layout, Precision, Transpose

__all__ = ["gemm", "try_gemm", "gemm_dev"]


def _as_slice(x, dtype, name, writable=False):
    if not isinstance(x, np.ndarray):
        raise TypeError(f"`{name}` must be a numpy array")
    if x.dtype != dtype:
        raise TypeError(f"`{name}` has dtype {x.dtype}, expected {np.dtype(dtype)}")
    if not x.flags["C_CONTIGUOUS"]:
        raise ValueError(f"`{name}` must be contiguous")
    if writable and not x.flags["WRITEABLE"]:
        raise ValueError(f"`{name}` must be writable")
    return x


def _ptr(x):
    return C.c_void_p(x.ctypes.data) if x.size else None


def try_gemm(layout, transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc,
             prec=Precision.Plain):
    """level3::try_gemm (src/level3.rs:68-103): validates, then computes
    C := alpha*op(A)*op(B) + beta*C in place. Returns None or a BlasError."""
    dt = c.dtype if isinstance(c, np.ndarray) else None
    if dt not in (np.float32, np.float64):
        raise TypeError("real gemm takes float32 or float64 slices")
    a = _as_slice(a, dt, "a")
    b = _as_slice(b, dt, "b")
    c = _as_slice(c, dt, "c", writable=True)
    lib = _lib.load()
    err = _lib.RbError()
    fn = lib.rb_sgemm_prec if dt == np.float32 else lib.rb_dgemm_prec
    st = fn(int(Layout(layout)), int(Transpose(transa)), int(Transpose(transb)), m, n, k, alpha,
            _ptr(a), lda, a.size, _ptr(b), ldb, b.size, beta, _ptr(c), ldc, c.size,
            int(Precision(prec)), C.byref(err))
    return _lib.raise_for(st, err)


def gemm(layout, transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc,
         prec=Precision.Plain):
    """level3::gemm (src/level3.rs:32-62): raises where rblas panics."""
    e = try_gemm(layout, transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, prec)
    if e is not None:
        raise e


def gemm_dev(layout, transa, transb, m, n, k, alpha, a_ptr, lda, b_ptr, ldb, beta, c_ptr, ldc,
             dtype, prec=Precision.Plain, stream=0):
    """Device-pointer GEMM: enqueue on `stream` (an int cudaStream_t handle)
    and return without synchronising. Pointers are ints (device addresses)."""
    lib = _lib.load()
    err = _lib.RbError()
    fn = lib.rb_sgemm_dev if np.dtype(dtype) == np.float32 else lib.rb_dgemm_dev
    st = fn(int(Layout(layout)), int(Transpose(transa)), int(Transpose(transb)), m, n, k, alpha,
            C.c_void_p(a_ptr), lda, C.c_void_p(b_ptr), ldb, beta, C.c_void_p(c_ptr), ldc,
            int(Precision(prec)), C.c_void_p(stream) if stream else None, C.byref(err))
    _lib.check(st, err)
