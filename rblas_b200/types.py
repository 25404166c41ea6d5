"""rblas's descriptor enums (src/types.rs:9-72), with the integer values the
C ABI uses (include/rblas_b200.h)."""
from enum import IntEnum


class Layout(IntEnum):
    """src/types.rs:9-14"""
    RowMajor = 0
    ColMajor = 1

    def strides(self, lda: int):
        """src/types.rs:20-25: (row_stride, col_stride) in elements."""
        return (lda, 1) if self is Layout.RowMajor else (1, lda)


class Transpose(IntEnum):
    """src/types.rs:30-37"""
    NoTrans = 0
    Trans = 1
    ConjTrans = 2

    def is_transposed(self) -> bool:
        """src/types.rs:42-44"""
        return self is not Transpose.NoTrans


class Uplo(IntEnum):
    """src/types.rs:49-54"""
    Upper = 0
    Lower = 1


class Side(IntEnum):
    """src/types.rs:58-63"""
    Left = 0
    Right = 1


class Diag(IntEnum):
    """src/types.rs:67-72"""
    NonUnit = 0
    Unit = 1


class Precision(IntEnum):
    """Arithmetic form of a GEMM call (no rblas counterpart: rblas has only
    the plain form). PLAIN is the drop-in."""
    Plain = 0
    Bf16x3 = 1
    Ozaki = 2
    Bf16x6 = 3
