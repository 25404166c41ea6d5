"""Batching and serving forms of rblas's gemm (level3::gemm, src/level3.rs:32-62)
on device-resident operands: the grouped persistent kernel and the serving
loop of librblas_b200.so (rb_gemm_grouped_dev, rb_server_*)."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from .types import Layout, Transpose

__all__ = ["Problem", "grouped_gemm", "grouped_gemm_bf16", "grouped_gemm_ozaki", "grouped_splits", "GroupedPlan", "Server", "autotune", "autotune_load",
           "autotune_reset"]


@dataclass
class Problem:
    """C := alpha*op(A)*op(B) + beta*C with device pointers (ints)."""
    dtype: object  # np.float32 / np.float64
    layout: int
    transa: int
    transb: int
    m: int
    n: int
    k: int
    alpha: float
    a: int
    lda: int
    b: int
    ldb: int
    beta: float
    c: int
    ldc: int

    def to_c(self) -> _lib.RbGemmProblem:
        return _lib.RbGemmProblem(
            0 if np.dtype(self.dtype) == np.float32 else 1, int(Layout(self.layout)),
            int(Transpose(self.transa)), int(Transpose(self.transb)), self.m, self.n, self.k,
            float(self.alpha), float(self.beta), C.c_void_p(self.a), self.lda, C.c_void_p(self.b),
            self.ldb, C.c_void_p(self.c), self.ldc)


def _array(problems):
    arr = (_lib.RbGemmProblem * len(problems))()
    for i, p in enumerate(problems):
        arr[i] = p.to_c() if isinstance(p, Problem) else p
    return arr


def grouped_gemm(problems, stream=0):
    """Run every problem in one grouped launch on `stream`."""
    arr = _array(problems)
    err = _lib.RbError()
    st = _lib.load().rb_gemm_grouped_dev(arr, len(problems), C.c_void_p(stream) if stream else None,
                                         C.byref(err))
    _lib.check(st, err)


def grouped_gemm_bf16(problems, form, stream=0):
    """Run f32 problems in a BF16-split form (Precision.Bf16x3 / Bf16x6) in
    one grouped launch on `stream` (rb_gemm_grouped_bf16_dev); each result
    equals its own call in that form."""
    arr = _array(problems)
    err = _lib.RbError()
    st = _lib.load().rb_gemm_grouped_bf16_dev(arr, len(problems), int(form), C.c_void_p(stream) if stream else None,
                                              C.byref(err))
    _lib.check(st, err)


def grouped_gemm_ozaki(problems, stream=0):
    """Run f64 problems in the Ozaki form in one grouped launch on `stream`
    (rb_gemm_grouped_ozaki_dev); each result equals its own Ozaki call."""
    arr = _array(problems)
    err = _lib.RbError()
    st = _lib.load().rb_gemm_grouped_ozaki_dev(arr, len(problems), C.c_void_p(stream) if stream else None,
                                               C.byref(err))
    _lib.check(st, err)


class GroupedPlan:
    """A grouped launch frozen into a CUDA graph (rb_gemm_grouped_plan_*):
    built once, replayed with launch(stream)."""

    def __init__(self, problems):
        self._lib = _lib.load()
        arr = _array(problems)
        h = C.c_void_p()
        err = _lib.RbError()
        st = self._lib.rb_gemm_grouped_plan_create(arr, len(problems), C.byref(h), C.byref(err))
        _lib.check(st, err)
        self._h = h

    def launch(self, stream=0):
        err = _lib.RbError()
        st = self._lib.rb_gemm_grouped_plan_launch(self._h, C.c_void_p(stream) if stream else None, C.byref(err))
        _lib.check(st, err)

    def close(self):
        if self._h:
            self._lib.rb_gemm_grouped_plan_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def _check(st):
    err = _lib.RbError()
    err.code = st
    _lib.check(st, err)


def autotune(cache_path: str | None = None) -> int:
    """Run the grouped kernel's split-K autotuner (rb_autotune_grouped) and
    install its table; returns the number of shape buckets timed."""
    n = C.c_int()
    st = _lib.load().rb_autotune_grouped(cache_path.encode() if cache_path else None, C.byref(n))
    _check(st)
    return n.value


def autotune_load(cache_path: str) -> None:
    st = _lib.load().rb_autotune_load(cache_path.encode())
    _check(st)


def autotune_reset() -> None:
    _lib.load().rb_autotune_reset()


def grouped_splits(p: Problem) -> int:
    """Split-K factor the grouped kernel uses for p (shape-only; 0 if invalid)."""
    q = p.to_c()
    return _lib.load().rb_gemm_grouped_splits(C.byref(q))


class Server:
    """The library's serving loop (rb_server_*): requests on device-resident
    inputs, results in server-owned HBM under a budget, continuous batching
    into grouped launches (grouped=True) or one launch per request."""

    def __init__(self, budget_bytes: int, max_batch: int = 256, grouped: bool = True):
        self._lib = _lib.load()
        h = C.c_void_p()
        st = self._lib.rb_server_create(budget_bytes, max_batch, int(grouped), C.byref(h))
        if st != 0:
            raise RuntimeError(f"rb_server_create failed: {self._lib.rb_status_string(st).decode()}")
        self._h = h

    def set_forms(self, f32_form=0, f64_form=0, f32_min_flop=0.0, f64_min_flop=0.0):
        """Run large requests in a precision form (rb_server_set_forms):
        f32 requests of >= f32_min_flop flop in f32_form (Precision.Bf16x3 /
        Bf16x6), f64 requests of >= f64_min_flop in f64_form (Precision.Ozaki)."""
        st = self._lib.rb_server_set_forms(self._h, int(f32_form), int(f64_form), float(f32_min_flop),
                                           float(f64_min_flop))
        if st != 0:
            raise RuntimeError(f"rb_server_set_forms failed: {self._lib.rb_status_string(st).decode()}")

    def submit(self, p: Problem) -> int:
        rid = C.c_uint64()
        q = p.to_c()
        st = self._lib.rb_server_submit(self._h, C.byref(q), C.byref(rid))
        if st != 0:
            raise RuntimeError(f"submit failed: {self._lib.rb_status_string(st).decode()}")
        return rid.value

    def wait(self, rid: int, timeout_us: int = -1):
        """-> (status, result_ptr, ldd, (enqueue_ns, admit_ns, finish_ns))."""
        d = C.c_void_p()
        ldd = C.c_size_t()
        t = _lib.RbRequestTimes()
        st = self._lib.rb_server_wait(self._h, rid, timeout_us, C.byref(d), C.byref(ldd), C.byref(t))
        return st, d.value, ldd.value, (t.enqueue_ns, t.admit_ns, t.finish_ns)

    def release(self, rid: int) -> int:
        return self._lib.rb_server_release(self._h, rid)

    def cancel(self, rid: int) -> int:
        """Cancel a still-queued request (rb_server_cancel): 0 when cancelled
        (its wait then reports RB_ERR_CANCELLED), RB_ERR_BUSY once admitted."""
        return self._lib.rb_server_cancel(self._h, rid)

    def run_trace(self, problems, arrival_ns):
        """Replay a trace natively; returns an (n, 3) uint64 array of
        (enqueue, admit, finish) ns and the status."""
        arr = _array(problems)
        arrivals = np.ascontiguousarray(arrival_ns, dtype=np.uint64)
        times = (_lib.RbRequestTimes * len(problems))()
        st = self._lib.rb_server_run_trace(self._h, arr, arrivals.ctypes.data_as(C.POINTER(C.c_uint64)),
                                           len(problems), times)
        out = np.array([(t.enqueue_ns, t.admit_ns, t.finish_ns) for t in times], dtype=np.uint64)
        return st, out

    def close(self):
        if self._h:
            self._lib.rb_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
