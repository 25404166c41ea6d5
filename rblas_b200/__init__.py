"""rblas_b200 -- a B200 (sm_100a) GEMM engine behind rblas's Level-3 API.

The product is the C ABI library librblas_b200.so (include/rblas_b200.h);
this package is its Python mirror of rblas's `level3` / `complex3` modules
(and of `level1` / `complex1` / `level2` / `complex2` around them), for hosts
and tests that call it from Python.
"""
from . import _lib, complex1, complex2, complex3, level1, level2, level3, serving
from .error import BlasError, BufferTooSmall, DeviceError, InvalidLeadingDim, ZeroStride
from .types import Diag, Layout, Precision, Side, Transpose, Uplo

__all__ = ["level1", "level2", "level3", "complex1", "complex2", "complex3", "serving", "Layout", "Transpose", "Uplo", "Side", "Diag", "Precision", "BlasError",
           "InvalidLeadingDim", "BufferTooSmall", "ZeroStride", "DeviceError", "launch_count",
           "device_error", "load_library"]


def load_library():
    return _lib.load()


def launch_count() -> int:
    """Kernels the library has launched since it was loaded."""
    return int(_lib.load().rb_launch_count())


def device_error(clear: bool = True):
    """(status, detail) of the current device's error word (synchronises)."""
    import ctypes as C
    d = C.c_uint32(0)
    st = _lib.load().rb_device_error(int(clear), C.byref(d))
    return int(st), int(d.value)
