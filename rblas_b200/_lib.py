"""ctypes binding of librblas_b200.so (include/rblas_b200.h).

The library is built in-tree (rblas_b200/_build.py). There is no CPU
fallback: if the shared library is missing or cannot be loaded, every call
raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

from .error import BlasError, BufferTooSmall, DeviceError, InvalidLeadingDim, ZeroStride

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "librblas_b200.so")

_lib = None
_lock = threading.Lock()


class RbError(C.Structure):
    _fields_ = [("code", C.c_int32), ("which", C.c_char), ("got", C.c_uint64),
                ("min_or_need", C.c_uint64), ("cuda_error", C.c_int32)]


class RbGemmProblem(C.Structure):
    _fields_ = [("dtype", C.c_int32), ("layout", C.c_int32), ("transa", C.c_int32),
                ("transb", C.c_int32), ("m", C.c_size_t), ("n", C.c_size_t), ("k", C.c_size_t),
                ("alpha", C.c_double), ("beta", C.c_double), ("a", C.c_void_p), ("lda", C.c_size_t),
                ("b", C.c_void_p), ("ldb", C.c_size_t), ("c", C.c_void_p), ("ldc", C.c_size_t)]


class RbRequestTimes(C.Structure):
    _fields_ = [("enqueue_ns", C.c_uint64), ("admit_ns", C.c_uint64), ("finish_ns", C.c_uint64)]


class RbComplex32(C.Structure):
    _fields_ = [("re", C.c_float), ("im", C.c_float)]


class RbComplex64(C.Structure):
    _fields_ = [("re", C.c_double), ("im", C.c_double)]


_sz, _i, _f, _d, _vp = C.c_size_t, C.c_int, C.c_float, C.c_double, C.c_void_p
_perr = C.POINTER(RbError)

# name -> (restype, argtypes)
SIGNATURES = {
    "rb_status_string": (C.c_char_p, [C.c_int32]),
    "rb_sgemm": (_i, [_i, _i, _i, _sz, _sz, _sz, _f, _vp, _sz, _sz, _vp, _sz, _sz, _f, _vp, _sz, _sz, _perr]),
    "rb_dgemm": (_i, [_i, _i, _i, _sz, _sz, _sz, _d, _vp, _sz, _sz, _vp, _sz, _sz, _d, _vp, _sz, _sz, _perr]),
    "rb_sgemm_prec": (_i, [_i, _i, _i, _sz, _sz, _sz, _f, _vp, _sz, _sz, _vp, _sz, _sz, _f, _vp, _sz, _sz, _i, _perr]),
    "rb_dgemm_prec": (_i, [_i, _i, _i, _sz, _sz, _sz, _d, _vp, _sz, _sz, _vp, _sz, _sz, _d, _vp, _sz, _sz, _i, _perr]),
    "rb_sgemm_dev": (_i, [_i, _i, _i, _sz, _sz, _sz, _f, _vp, _sz, _vp, _sz, _f, _vp, _sz, _i, _vp, _perr]),
    "rb_dgemm_dev": (_i, [_i, _i, _i, _sz, _sz, _sz, _d, _vp, _sz, _vp, _sz, _d, _vp, _sz, _i, _vp, _perr]),
    "rb_cgemm": (_i, [_i, _i, _sz, _sz, _sz, RbComplex32, _vp, _sz, _sz, _vp, _sz, _sz, RbComplex32, _vp, _sz, _sz, _i, _perr]),
    "rb_zgemm": (_i, [_i, _i, _sz, _sz, _sz, RbComplex64, _vp, _sz, _sz, _vp, _sz, _sz, RbComplex64, _vp, _sz, _sz, _i, _perr]),
    "rb_cgemm_dev": (_i, [_i, _i, _sz, _sz, _sz, RbComplex32, _vp, _sz, _vp, _sz, RbComplex32, _vp, _sz, _i, _vp, _perr]),
    "rb_zgemm_dev": (_i, [_i, _i, _sz, _sz, _sz, RbComplex64, _vp, _sz, _vp, _sz, RbComplex64, _vp, _sz, _i, _vp, _perr]),
    "rb_ssyrk": (_i, [_i, _i, _sz, _sz, _f, _vp, _sz, _sz, _f, _vp, _sz, _sz, _perr]),
    "rb_dsyrk": (_i, [_i, _i, _sz, _sz, _d, _vp, _sz, _sz, _d, _vp, _sz, _sz, _perr]),
    "rb_ssymm": (_i, [_i, _i, _sz, _sz, _f, _vp, _sz, _sz, _vp, _sz, _sz, _f, _vp, _sz, _sz, _perr]),
    "rb_dsymm": (_i, [_i, _i, _sz, _sz, _d, _vp, _sz, _sz, _vp, _sz, _sz, _d, _vp, _sz, _sz, _perr]),
    "rb_csymm": (_i, [_i, _i, _sz, _sz, RbComplex32, _vp, _sz, _sz, _vp, _sz, _sz, RbComplex32, _vp, _sz, _sz, _perr]),
    "rb_zsymm": (_i, [_i, _i, _sz, _sz, RbComplex64, _vp, _sz, _sz, _vp, _sz, _sz, RbComplex64, _vp, _sz, _sz, _perr]),
    "rb_chemm": (_i, [_i, _i, _sz, _sz, RbComplex32, _vp, _sz, _sz, _vp, _sz, _sz, RbComplex32, _vp, _sz, _sz, _perr]),
    "rb_zhemm": (_i, [_i, _i, _sz, _sz, RbComplex64, _vp, _sz, _sz, _vp, _sz, _sz, RbComplex64, _vp, _sz, _sz, _perr]),
    "rb_strsm": (_i, [_i, _i, _i, _i, _sz, _sz, _f, _vp, _sz, _sz, _vp, _sz, _sz, _perr]),
    "rb_dtrsm": (_i, [_i, _i, _i, _i, _sz, _sz, _d, _vp, _sz, _sz, _vp, _sz, _sz, _perr]),
    "rb_ctrsm": (_i, [_i, _i, _i, _i, _sz, _sz, RbComplex32, _vp, _sz, _sz, _vp, _sz, _sz, _perr]),
    "rb_ztrsm": (_i, [_i, _i, _i, _i, _sz, _sz, RbComplex64, _vp, _sz, _sz, _vp, _sz, _sz, _perr]),
    "rb_strmm": (_i, [_i, _i, _i, _i, _sz, _sz, _f, _vp, _sz, _sz, _vp, _sz, _sz, _perr]),
    "rb_dtrmm": (_i, [_i, _i, _i, _i, _sz, _sz, _d, _vp, _sz, _sz, _vp, _sz, _sz, _perr]),
    "rb_ctrmm": (_i, [_i, _i, _i, _i, _sz, _sz, RbComplex32, _vp, _sz, _sz, _vp, _sz, _sz, _perr]),
    "rb_ztrmm": (_i, [_i, _i, _i, _i, _sz, _sz, RbComplex64, _vp, _sz, _sz, _vp, _sz, _sz, _perr]),
    "rb_dtrmm_dev": (_i, [_i, _i, _i, _i, _sz, _sz, _d, _vp, _sz, _vp, _sz, _vp, _perr]),
    "rb_sgemv": (_i, [_i, _i, _sz, _sz, _f, _vp, _sz, _sz, _vp, _sz, _sz, _f, _vp, _sz, _sz, _perr]),
    "rb_sgemv_dev": (_i, [_i, _i, _sz, _sz, _f, _vp, _sz, _vp, _sz, _f, _vp, _sz, _vp, _perr]),
    "rb_dgemv": (_i, [_i, _i, _sz, _sz, _d, _vp, _sz, _sz, _vp, _sz, _sz, _d, _vp, _sz, _sz, _perr]),
    "rb_dgemv_dev": (_i, [_i, _i, _sz, _sz, _d, _vp, _sz, _vp, _sz, _d, _vp, _sz, _vp, _perr]),
    "rb_cgemv": (_i, [_i, _i, _sz, _sz, RbComplex32, _vp, _sz, _sz, _vp, _sz, _sz, RbComplex32, _vp, _sz, _sz, _perr]),
    "rb_cgemv_dev": (_i, [_i, _i, _sz, _sz, RbComplex32, _vp, _sz, _vp, _sz, RbComplex32, _vp, _sz, _vp, _perr]),
    "rb_zgemv": (_i, [_i, _i, _sz, _sz, RbComplex64, _vp, _sz, _sz, _vp, _sz, _sz, RbComplex64, _vp, _sz, _sz, _perr]),
    "rb_zgemv_dev": (_i, [_i, _i, _sz, _sz, RbComplex64, _vp, _sz, _vp, _sz, RbComplex64, _vp, _sz, _vp, _perr]),
    "rb_sger": (_i, [_i, _sz, _sz, _f, _vp, _sz, _sz, _vp, _sz, _sz, _vp, _sz, _sz, _perr]),
    "rb_sger_dev": (_i, [_i, _sz, _sz, _f, _vp, _sz, _vp, _sz, _vp, _sz, _vp, _perr]),
    "rb_dger": (_i, [_i, _sz, _sz, _d, _vp, _sz, _sz, _vp, _sz, _sz, _vp, _sz, _sz, _perr]),
    "rb_dger_dev": (_i, [_i, _sz, _sz, _d, _vp, _sz, _vp, _sz, _vp, _sz, _vp, _perr]),
    "rb_cgeru": (_i, [_i, _sz, _sz, RbComplex32, _vp, _sz, _sz, _vp, _sz, _sz, _vp, _sz, _sz, _perr]),
    "rb_cgeru_dev": (_i, [_i, _sz, _sz, RbComplex32, _vp, _sz, _vp, _sz, _vp, _sz, _vp, _perr]),
    "rb_zgeru": (_i, [_i, _sz, _sz, RbComplex64, _vp, _sz, _sz, _vp, _sz, _sz, _vp, _sz, _sz, _perr]),
    "rb_zgeru_dev": (_i, [_i, _sz, _sz, RbComplex64, _vp, _sz, _vp, _sz, _vp, _sz, _vp, _perr]),
    "rb_cgerc": (_i, [_i, _sz, _sz, RbComplex32, _vp, _sz, _sz, _vp, _sz, _sz, _vp, _sz, _sz, _perr]),
    "rb_cgerc_dev": (_i, [_i, _sz, _sz, RbComplex32, _vp, _sz, _vp, _sz, _vp, _sz, _vp, _perr]),
    "rb_zgerc": (_i, [_i, _sz, _sz, RbComplex64, _vp, _sz, _sz, _vp, _sz, _sz, _vp, _sz, _sz, _perr]),
    "rb_zgerc_dev": (_i, [_i, _sz, _sz, RbComplex64, _vp, _sz, _vp, _sz, _vp, _sz, _vp, _perr]),
    "rb_dtrsm_dev": (_i, [_i, _i, _i, _i, _sz, _sz, _d, _vp, _sz, _vp, _sz, _vp, _perr]),
    "rb_strsm_batched_dev": (_i, [_i, _i, _i, _i, _sz, _sz, C.c_float, _vp, _sz, _sz, _vp, _sz, _sz, _sz, _vp,
                                  _perr]),
    "rb_dtrsm_batched_dev": (_i, [_i, _i, _i, _i, _sz, _sz, _d, _vp, _sz, _sz, _vp, _sz, _sz, _sz, _vp, _perr]),
    "rb_dgemm_ozaki_noalloc": (_i, [_i, _i, _i, _sz, _sz, _sz, _d, _vp, _sz, _vp, _sz, _d, _vp, _sz, _vp, _perr]),
    "rb_gemm_grouped_dev": (_i, [C.POINTER(RbGemmProblem), _sz, _vp, _perr]),
    "rb_gemm_grouped_splits": (_i, [C.POINTER(RbGemmProblem)]),
    "rb_gemm_grouped_ozaki_dev": (_i, [C.POINTER(RbGemmProblem), _sz, _vp, _perr]),
    "rb_gemm_grouped_bf16_dev": (_i, [C.POINTER(RbGemmProblem), _sz, _i, _vp, _perr]),
    "rb_gemm_grouped_plan_create": (_i, [C.POINTER(RbGemmProblem), _sz, C.POINTER(C.c_void_p), _perr]),
    "rb_gemm_grouped_plan_launch": (_i, [_vp, _vp, _perr]),
    "rb_gemm_grouped_plan_destroy": (_i, [_vp]),
    "rb_autotune_grouped": (_i, [C.c_char_p, C.POINTER(C.c_int)]),
    "rb_autotune_load": (_i, [C.c_char_p]),
    "rb_autotune_reset": (_i, []),
    "rb_server_create": (_i, [_sz, _i, _i, C.POINTER(C.c_void_p)]),
    "rb_server_set_forms": (_i, [_vp, _i, _i, _d, _d]),
    "rb_server_submit": (_i, [_vp, C.POINTER(RbGemmProblem), C.POINTER(C.c_uint64)]),
    "rb_server_wait": (_i, [_vp, C.c_uint64, C.c_int64, C.POINTER(C.c_void_p), C.POINTER(C.c_size_t),
                            C.POINTER(RbRequestTimes)]),
    "rb_server_release": (_i, [_vp, C.c_uint64]),
    "rb_server_cancel": (_i, [_vp, C.c_uint64]),
    "rb_server_destroy": (_i, [_vp]),
    "rb_server_run_trace": (_i, [_vp, C.POINTER(RbGemmProblem), C.POINTER(C.c_uint64), _sz,
                                 C.POINTER(RbRequestTimes)]),
    "rb_set_ozaki_slices": (_i, [_i]),
    "rb_get_ozaki_slices": (_i, []),
    "rb_launch_count": (C.c_uint64, []),
    "rb_device_error": (_i, [_i, C.POINTER(C.c_uint32)]),
    "rb_probe_wait_timeout": (_i, [C.POINTER(C.c_uint32)]),
    "rb_num_threads": (C.c_size_t, []),
    "rb_device_alloc_count": (C.c_uint64, []),
    "rb_debug_inject": (_i, [_i, C.c_uint32, _i]),
    "rb_release_cached_memory": (None, []),
    "rb_set_scratch_cache_bytes": (None, [_sz]),
    "rb_probe_fma_peak_tflops": (C.c_double, [_i, _i]),
    "rb_probe_tensor_peak_tflops": (C.c_double, [_i, _i]),
    "rb_kernel_timing_enable": (None, [_i]),
    "rb_kernel_timing_report": (_i, [C.c_char_p, _sz]),
}


def _level1_signatures():
    """Level 1 (include/rblas_b200.h): host slices carry a length after each
    vector; the _dev forms take a stream instead. Reductions write *result."""
    sig = {}
    for p, t in (("s", _f), ("d", _d)):
        sig[f"rb_{p}axpy"] = (_i, [_sz, t, _vp, _sz, _sz, _vp, _sz, _sz, _perr])
        sig[f"rb_{p}axpy_dev"] = (_i, [_sz, t, _vp, _sz, _vp, _sz, _vp, _perr])
        sig[f"rb_{p}scal"] = (_i, [_sz, t, _vp, _sz, _sz, _perr])
        sig[f"rb_{p}scal_dev"] = (_i, [_sz, t, _vp, _sz, _vp, _perr])
        for name in ("copy", "swap"):
            sig[f"rb_{p}{name}"] = (_i, [_sz, _vp, _sz, _sz, _vp, _sz, _sz, _perr])
            sig[f"rb_{p}{name}_dev"] = (_i, [_sz, _vp, _sz, _vp, _sz, _vp, _perr])
        sig[f"rb_{p}dot"] = (_i, [_sz, _vp, _sz, _sz, _vp, _sz, _sz, _vp, _perr])
        sig[f"rb_{p}dot_dev"] = (_i, [_sz, _vp, _sz, _vp, _sz, _vp, _vp, _perr])
        for name in ("asum", "nrm2"):
            sig[f"rb_{p}{name}"] = (_i, [_sz, _vp, _sz, _sz, _vp, _perr])
            sig[f"rb_{p}{name}_dev"] = (_i, [_sz, _vp, _sz, _vp, _vp, _perr])
    for p, n, ct in (("c", "sc", RbComplex32), ("z", "dz", RbComplex64)):
        sig[f"rb_{p}axpy"] = (_i, [_sz, ct, _vp, _sz, _sz, _vp, _sz, _sz, _perr])
        sig[f"rb_{p}axpy_dev"] = (_i, [_sz, ct, _vp, _sz, _vp, _sz, _vp, _perr])
        sig[f"rb_{p}scal"] = (_i, [_sz, ct, _vp, _sz, _sz, _perr])
        sig[f"rb_{p}scal_dev"] = (_i, [_sz, ct, _vp, _sz, _vp, _perr])
        for name in ("dotu", "dotc"):
            sig[f"rb_{p}{name}"] = (_i, [_sz, _vp, _sz, _sz, _vp, _sz, _sz, _vp, _perr])
            sig[f"rb_{p}{name}_dev"] = (_i, [_sz, _vp, _sz, _vp, _sz, _vp, _vp, _perr])
        sig[f"rb_{n}nrm2"] = (_i, [_sz, _vp, _sz, _sz, _vp, _perr])
        sig[f"rb_{n}nrm2_dev"] = (_i, [_sz, _vp, _sz, _vp, _vp, _perr])
    return sig


SIGNATURES.update(_level1_signatures())


def load():
    """Load (once) and return the CDLL. Raises if the library is absent."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise ImportError(
                    f"{LIB_PATH} is missing: build it with `python -m rblas_b200._build` "
                    "(there is no CPU fallback)")
            lib = C.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(lib, name, None)
                if fn is None:
                    continue
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


def exported_symbols():
    lib = load()
    return [n for n in SIGNATURES if hasattr(lib, n)]


def raise_for(status: int, err: RbError):
    """Map an rb_status + rb_error to the matching BlasError."""
    if status == 0:
        return None
    which = err.which.decode() if err.which else ""
    if status == 1:
        return InvalidLeadingDim(which, int(err.got), int(err.min_or_need))
    if status == 2:
        return BufferTooSmall(which, int(err.got), int(err.min_or_need))
    if status == 3:
        return ZeroStride(which)
    msg = load().rb_status_string(status).decode()
    detail = int(err.cuda_error) if status == 6 else int(err.got)
    return DeviceError(status, msg, detail)


def check(status: int, err: RbError):
    e = raise_for(status, err)
    if e is not None:
        raise e
