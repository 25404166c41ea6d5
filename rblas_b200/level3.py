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

__all__ = ["num_threads", "gemm", "try_gemm", "gemm_dev", "syrk", "symm", "trsm"]


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


def num_threads():
    """level3::num_threads (src/level3.rs:11-17): the parallel width of the
    GEMM path -- the current device's SM count (one CTA per SM in every
    persistent GEMM kernel); 1 when no device is usable (like rayon's pool
    size, never 0)."""
    return int(_lib.load().rb_num_threads())


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


def _real_fn(lib, dt, name):
    return getattr(lib, ("rb_s" if dt == np.float32 else "rb_d") + name)


def _dtype_of(c):
    dt = c.dtype if isinstance(c, np.ndarray) else None
    if dt not in (np.float32, np.float64):
        raise TypeError("real routines take float32 or float64 slices")
    return dt


def syrk(uplo, trans, n, k, alpha, a, lda, beta, c, ldc):
    """level3::syrk (src/level3.rs:236-294): C := alpha*op(A)*op(A)^T + beta*C
    on the `uplo` triangle of the n x n C (op(A) is n x k)."""
    from .types import Uplo
    dt = _dtype_of(c)
    a = _as_slice(a, dt, "a")
    c = _as_slice(c, dt, "c", writable=True)
    lib = _lib.load()
    err = _lib.RbError()
    st = _real_fn(lib, dt, "syrk")(int(Uplo(uplo)), int(Transpose(trans)), n, k, alpha, _ptr(a), lda,
                                   a.size, beta, _ptr(c), ldc, c.size, C.byref(err))
    _lib.check(st, err)


def symm(side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc):
    """level3::symm (src/level3.rs:301-354): A symmetric (uplo triangle
    stored); C := alpha*A*B + beta*C (Left) or alpha*B*A + beta*C (Right)."""
    from .types import Side, Uplo
    dt = _dtype_of(c)
    a = _as_slice(a, dt, "a")
    b = _as_slice(b, dt, "b")
    c = _as_slice(c, dt, "c", writable=True)
    lib = _lib.load()
    err = _lib.RbError()
    st = _real_fn(lib, dt, "symm")(int(Side(side)), int(Uplo(uplo)), m, n, alpha, _ptr(a), lda, a.size,
                                   _ptr(b), ldb, b.size, beta, _ptr(c), ldc, c.size, C.byref(err))
    _lib.check(st, err)


def trsm(side, uplo, trans, diag, m, n, alpha, a, lda, b, ldb):
    """level3::trsm (src/level3.rs:390-437): solve op(A)*X = alpha*B (Left)
    or X*op(A) = alpha*B (Right) in place of B."""
    from .types import Diag, Side, Uplo
    dt = _dtype_of(b)
    a = _as_slice(a, dt, "a")
    b = _as_slice(b, dt, "b", writable=True)
    lib = _lib.load()
    err = _lib.RbError()
    st = _real_fn(lib, dt, "trsm")(int(Side(side)), int(Uplo(uplo)), int(Transpose(trans)),
                                   int(Diag(diag)), m, n, alpha, _ptr(a), lda, a.size, _ptr(b), ldb,
                                   b.size, C.byref(err))
    _lib.check(st, err)


def trsm_dev(side, uplo, trans, diag, m, n, alpha, a_ptr, lda, b_ptr, ldb, stream=0):
    """f64 trsm on device pointers (rb_dtrsm_dev), in place of B; enqueued
    on `stream`, no synchronisation."""
    from .types import Diag, Side, Uplo
    lib = _lib.load()
    err = _lib.RbError()
    st = lib.rb_dtrsm_dev(int(Side(side)), int(Uplo(uplo)), int(Transpose(trans)), int(Diag(diag)), m, n, alpha,
                          C.c_void_p(a_ptr), lda, C.c_void_p(b_ptr), ldb, C.c_void_p(stream) if stream else None,
                          C.byref(err))
    _lib.check(st, err)


def trsm_batched_dev(side, uplo, trans, diag, m, n, alpha, a_ptr, lda, stride_a, b_ptr, ldb, stride_b,
                     batch, dtype, stream=0):
    """Batched trsm on device pointers (rb_?trsm_batched_dev): problem i is
    trsm(side, uplo, trans, diag, m, n, alpha, A_i, lda, B_i, ldb) with
    A_i = a + i*stride_a, B_i = b + i*stride_b (elements). Enqueued on
    `stream`, no synchronisation."""
    from .types import Diag, Side, Uplo
    lib = _lib.load()
    err = _lib.RbError()
    fn = lib.rb_strsm_batched_dev if np.dtype(dtype) == np.float32 else lib.rb_dtrsm_batched_dev
    st = fn(int(Side(side)), int(Uplo(uplo)), int(Transpose(trans)), int(Diag(diag)), m, n, alpha,
            C.c_void_p(a_ptr), lda, stride_a, C.c_void_p(b_ptr), ldb, stride_b, batch,
            C.c_void_p(stream) if stream else None, C.byref(err))
    _lib.check(st, err)


def trmm(side, uplo, trans, diag, m, n, alpha, a, lda, b, ldb):
    """Triangular multiply in place of B: B := alpha*op(A)*B (Left) or
    alpha*B*op(A) (Right), A triangular. No rblas counterpart (its README
    lists trmm as remaining Level 3); arguments as level3::trsm."""
    from .types import Diag, Side, Uplo
    dt = _dtype_of(b)
    a = _as_slice(a, dt, "a")
    b = _as_slice(b, dt, "b", writable=True)
    err = _lib.RbError()
    st = _real_fn(_lib.load(), dt, "trmm")(int(Side(side)), int(Uplo(uplo)), int(Transpose(trans)),
                                           int(Diag(diag)), m, n, alpha, _ptr(a), lda, a.size, _ptr(b), ldb, b.size,
                                           C.byref(err))
    _lib.check(st, err)
