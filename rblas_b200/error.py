"""rblas's BlasError (src/error.rs:15-57) plus the GPU library's own
failure kinds, raised or returned like the Rust API: the checked (`try_*`)
functions return the error, the others raise it (rblas panics)."""
from __future__ import annotations


class BlasError(Exception):
    """Base class; `code` is the C ABI's rb_status."""
    code = -1

    def __eq__(self, other):
        return type(self) is type(other) and self.args == other.args

    def __hash__(self):
        return hash((type(self), self.args))


class InvalidLeadingDim(BlasError):
    """src/error.rs:17-24"""
    code = 1

    def __init__(self, which: str, got: int, min: int):
        super().__init__(which, got, min)
        self.which, self.got, self.min = which, got, min

    def __str__(self):
        # src/error.rs:44-47
        return f"invalid leading dimension for `{self.which}`: got {self.got}, need ≥ {self.min}"


class BufferTooSmall(BlasError):
    """src/error.rs:26-33"""
    code = 2

    def __init__(self, which: str, got: int, need: int):
        super().__init__(which, got, need)
        self.which, self.got, self.need = which, got, need

    def __str__(self):
        # src/error.rs:48-51
        return f"buffer `{self.which}` too small: got {self.got} elements, need ≥ {self.need}"


class ZeroStride(BlasError):
    """src/error.rs:35-38"""
    code = 3

    def __init__(self, which: str):
        super().__init__(which)
        self.which = which

    def __str__(self):
        return f"stride for `{self.which}` must be positive (got 0)"


class DeviceError(BlasError):
    """A failure of the GPU path itself (CUDA error, timeout, unsupported form)."""

    def __init__(self, code: int, message: str, detail: int = 0):
        super().__init__(code, message, detail)
        self.code, self.message, self.detail = code, message, detail

    def __str__(self):
        return f"{self.message} (status {self.code}, detail {self.detail:#x})"
