"""CPU tests of the C-ABI boundary: the library loads, exports every symbol
include/rblas_b200.h declares, and the host-side validation reproduces
rblas's try_gemm error contract (src/level3.rs:68-140) -- none of these
calls reach the GPU."""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np
import pytest

import rblas_b200 as rb
from rblas_b200 import _lib, level3
from rblas_b200.types import Layout, Transpose
from tests.golden_runner import load_cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "rblas_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(rb_[a-z0-9_]+)\s*\(", src)))


def test_library_builds_and_loads():
    lib = _lib.load()
    assert lib is not None


def test_every_declared_symbol_is_exported():
    lib = _lib.load()
    missing = [f for f in header_functions() if not hasattr(lib, f)]
    assert not missing, f"declared but not exported: {missing}"


def test_every_declared_symbol_has_a_binding():
    missing = [f for f in header_functions() if f not in _lib.SIGNATURES]
    assert not missing, f"no ctypes signature for: {missing}"


def test_status_strings():
    lib = _lib.load()
    assert lib.rb_status_string(0) == b"ok"
    assert lib.rb_status_string(2) == b"buffer too small"


def test_try_gemm_error_contract_matches_reference():
    """src/level3.rs:567-640 with the exact error fields."""
    meta, _ = load_cases()["try_gemm_errors"]
    m, n, k = meta["m"], meta["n"], meta["k"]
    for call in meta["calls"][1:]:
        a = np.ones(call["a_len"])
        b = np.ones(call["b_len"])
        c = np.zeros(call["c_len"])
        e = level3.try_gemm(Layout.ColMajor, Transpose.NoTrans, Transpose.NoTrans, m, n, k, 1.0,
                            a, call["lda"], b, call["ldb"], 0.0, c, call["ldc"])
        w = call["want"]
        if w["code"] == 1:
            assert e == rb.InvalidLeadingDim(w["which"], w["got"], w["min_or_need"])
            assert str(e) == "invalid leading dimension for `a`: got 3, need ≥ 4"
        else:
            assert e == rb.BufferTooSmall(w["which"], w["got"], w["min_or_need"])


@pytest.mark.parametrize("layout", [Layout.RowMajor, Layout.ColMajor])
def test_validation_order_and_fields(layout):
    """a, b, c in order; InvalidLeadingDim before BufferTooSmall; stored
    shapes follow the transpose (src/level3.rs:86-98, 121-138)."""
    m, n, k = 5, 7, 3
    ta, tb = Transpose.Trans, Transpose.NoTrans
    # stored A is k x m; row-major min lead = cols = m, col-major = rows = k
    min_a = m if layout == Layout.RowMajor else k
    a = np.zeros(100)
    b = np.zeros(100)
    c = np.zeros(100)
    e = level3.try_gemm(layout, ta, tb, m, n, k, 1.0, a, min_a - 1, b, 100, 0.0, c, 100)
    assert e == rb.InvalidLeadingDim("a", min_a - 1, min_a)
    # bad b and bad c: a is reported first only when a is bad
    min_b = n if layout == Layout.RowMajor else k
    e = level3.try_gemm(layout, ta, tb, m, n, k, 1.0, a, min_a, b, min_b - 1, 0.0, c, 0)
    assert e == rb.InvalidLeadingDim("b", min_b - 1, min_b)
    # buffer too small on c: need = (n-1)*ldc + m (col) / (m-1)*ldc + n (row)
    ldc = 9
    need = (n - 1) * ldc + m if layout == Layout.ColMajor else (m - 1) * ldc + n
    cs = np.zeros(need - 1)
    e = level3.try_gemm(layout, ta, tb, m, n, k, 1.0, a, min_a, b, min_b, 0.0, cs, ldc)
    assert e == rb.BufferTooSmall("c", need - 1, need)


def test_zero_dims_are_valid_and_touch_nothing():
    """check_matrix returns Ok for zero dims; gemm_contig returns before beta."""
    c = np.full(4, np.nan)
    e = level3.try_gemm(Layout.ColMajor, Transpose.NoTrans, Transpose.NoTrans, 0, 4, 3, 1.0,
                        np.zeros(0), 0, np.zeros(12), 3, 0.0, c, 1)
    assert e is None and np.all(np.isnan(c))


def test_invalid_enum_rejected_by_the_c_layer():
    import ctypes as C
    lib = _lib.load()
    err = _lib.RbError()
    buf = np.zeros(4)
    p = C.c_void_p(buf.ctypes.data)
    st = lib.rb_dgemm(7, 0, 0, 2, 2, 2, 1.0, p, 2, 4, p, 2, 4, 0.0, p, 2, 4, C.byref(err))
    assert st == 4 and err.code == 4
    with pytest.raises(ValueError):
        level3.try_gemm(7, 0, 0, 2, 2, 2, 1.0, buf, 2, buf, 2, 0.0, buf, 2)


def test_num_threads_mirrors_level3():
    """level3::num_threads: the SM count on a GPU, 1 where no device is usable
    (rblas's rayon pool size is never 0, and callers divide by it)."""
    from rblas_b200 import level3
    try:
        import torch
        sms = torch.cuda.get_device_properties(0).multi_processor_count if torch.cuda.is_available() else 1
    except ImportError:
        sms = None
    got = level3.num_threads()
    assert got == sms if sms is not None else got >= 1


def test_debug_inject_argument_checks():
    """rb_debug_inject rejects unknown kinds, negative counts and a zero
    device word before touching any device."""
    lib = _lib.load()
    assert lib.rb_debug_inject(0, 0, 0) == 4
    assert lib.rb_debug_inject(3, 1, 1) == 4
    assert lib.rb_debug_inject(1, 0, -1) == 4
    assert lib.rb_debug_inject(2, 0, 0) == 4
    assert lib.rb_debug_inject(1, 0, 2) == 0  # arm two failures ...
    assert lib.rb_debug_inject(1, 0, 0) == 0  # ... and clear them again
    assert lib.rb_device_alloc_count() >= 0


def test_noalloc_rejects_null_pointers_before_any_device_work():
    """rb_dgemm_ozaki_noalloc, like rb_dgemm_dev, rejects a null a or b (k > 0)
    or a null c with RB_ERR_INVALID_ARG; it checks before touching a device,
    so this runs without one."""
    lib = _lib.load()
    buf = np.zeros(64, dtype=np.float64)
    p = C.c_void_p(buf.ctypes.data)
    for a, b, c in ((None, p, p), (p, None, p), (p, p, None)):
        err = _lib.RbError()
        st = lib.rb_dgemm_ozaki_noalloc(1, 0, 0, 4, 4, 4, 1.0, a, 4, b, 4, 0.0, c, 4, None, C.byref(err))
        assert st == 4 and err.code == 4
    # k == 0 never reads a or b: only c must be given
    err = _lib.RbError()
    st = lib.rb_dgemm_ozaki_noalloc(1, 0, 0, 4, 4, 0, 1.0, None, 4, None, 1, 0.0, None, 4, None, C.byref(err))
    assert st == 4
    # leading dimensions are still checked first, as in check_matrix
    err = _lib.RbError()
    st = lib.rb_dgemm_ozaki_noalloc(1, 0, 0, 4, 4, 4, 1.0, None, 3, p, 4, 0.0, p, 4, None, C.byref(err))
    assert st == 1 and err.which == b"a"


def test_noalloc_scratch_limit_is_overflow_safe():
    """Sizes whose scratch bytes would wrap a 64-bit product are rejected with
    RB_ERR_SCRATCH_LIMIT before any device work (no device needed)."""
    lib = _lib.load()
    buf = np.zeros(8, dtype=np.float64)
    p = C.c_void_p(buf.ctypes.data)
    big = 2 ** 31 - 1
    err = _lib.RbError()
    st = lib.rb_dgemm_ozaki_noalloc(1, 0, 0, big, big, big, 1.0, p, big, p, big, 0.0, p, big, None, C.byref(err))
    assert st == 12 and err.got > err.min_or_need == (64 << 20) + (64 << 10)


def test_grouped_ozaki_rejects_non_f64_entries_before_any_device_work():
    """rb_gemm_grouped_ozaki_dev takes f64 problems only: an f32 entry is
    RB_ERR_UNSUPPORTED with its index, a null C is RB_ERR_INVALID_ARG; both
    are found before anything is enqueued (no device needed)."""
    lib = _lib.load()
    buf = np.zeros(64, dtype=np.float64)
    p = buf.ctypes.data
    arr = (_lib.RbGemmProblem * 2)()
    for i in range(2):
        arr[i] = _lib.RbGemmProblem(1, 1, 0, 0, 4, 4, 4, 1.0, 0.0, C.c_void_p(p), 4, C.c_void_p(p), 4,
                                    C.c_void_p(p), 4)
    arr[1].dtype = 0
    err = _lib.RbError()
    assert lib.rb_gemm_grouped_ozaki_dev(arr, 2, None, C.byref(err)) == 5 and err.got == 1
    arr[1].dtype = 1
    arr[0].c = None
    err = _lib.RbError()
    assert lib.rb_gemm_grouped_ozaki_dev(arr, 2, None, C.byref(err)) == 4 and err.got == 0


def test_grouped_bf16_rejects_bad_tables_before_any_device_work():
    """rb_gemm_grouped_bf16_dev: a form other than BF16X3/BF16X6 is
    RB_ERR_INVALID_ARG, an f64 entry RB_ERR_UNSUPPORTED with its index."""
    lib = _lib.load()
    buf = np.zeros(64, dtype=np.float32)
    p = buf.ctypes.data
    arr = (_lib.RbGemmProblem * 2)()
    for i in range(2):
        arr[i] = _lib.RbGemmProblem(0, 1, 0, 0, 4, 4, 4, 1.0, 0.0, C.c_void_p(p), 4, C.c_void_p(p), 4,
                                    C.c_void_p(p), 4)
    err = _lib.RbError()
    assert lib.rb_gemm_grouped_bf16_dev(arr, 2, 2, None, C.byref(err)) == 4  # Ozaki is not a BF16 form
    arr[1].dtype = 1
    err = _lib.RbError()
    assert lib.rb_gemm_grouped_bf16_dev(arr, 2, 3, None, C.byref(err)) == 5 and err.got == 1


def test_ctypes_signatures_match_the_header():
    """Every ctypes binding takes as many arguments as its C declaration, and
    each argument is passed in the declared width: pointers as pointers,
    size_t as c_size_t, float / double as c_float / c_double, the enums and
    ints as 32-bit ints, complex scalars as their two-field structures."""
    from tests.test_rust_ffi_cpu import header_functions as header_params

    scalars = {
        "size_t": (C.c_size_t,), "float": (C.c_float,), "double": (C.c_double,),
        "int": (C.c_int, C.c_int32), "int32_t": (C.c_int, C.c_int32), "uint32_t": (C.c_uint32,),
        "uint64_t": (C.c_uint64,), "int64_t": (C.c_int64,),
        "rb_complex32": (_lib.RbComplex32,), "rb_complex64": (_lib.RbComplex64,),
    }
    for e in ("rb_layout", "rb_transpose", "rb_uplo", "rb_side", "rb_diag", "rb_precision"):
        scalars[e] = (C.c_int, C.c_int32)
    for name, cparams in header_params().items():
        _, args = _lib.SIGNATURES[name]
        assert len(args) == len(cparams), f"{name}: {len(args)} ctypes arguments, {len(cparams)} in the header"
        for a, c in zip(args, cparams):
            if "*" in c:
                assert a in (C.c_void_p, C.c_char_p) or issubclass(a, C._Pointer), f"{name}: `{c}` as {a}"
            else:
                base = c.replace("const ", "").split()[0]
                assert a in scalars[base], f"{name}: `{c}` as {a}"


def test_ctypes_return_types_match_the_header():
    """Each binding's restype is the C declaration's return type."""
    from tests.test_rust_ffi_cpu import header_functions as header_params

    text = re.sub(r"/\*.*?\*/", "", open(os.path.join(ROOT, "include", "rblas_b200.h")).read(), flags=re.S)
    expect = {"rb_status": (C.c_int, C.c_int32), "int": (C.c_int, C.c_int32), "int32_t": (C.c_int, C.c_int32),
              "size_t": (C.c_size_t,), "uint64_t": (C.c_uint64,), "uint32_t": (C.c_uint32,),
              "double": (C.c_double,), "void": (None,), "const char*": (C.c_char_p,)}
    seen = 0
    for m in re.finditer(r"^\s*((?:const\s+)?\w+\s*\**)\s*(rb_\w+)\s*\(", text, re.M):
        ret, name = " ".join(m.group(1).replace("*", " * ").split()).replace(" *", "*"), m.group(2)
        if ret.startswith("typedef"):
            continue
        res, _ = _lib.SIGNATURES[name]
        assert res in expect[ret], f"{name}: returns `{ret}`, bound as {res}"
        seen += 1
    assert seen == len(header_params())


def test_no_cpu_fallback_without_a_device():
    """On a host without a GPU a GEMM call raises instead of computing
    anywhere else, and leaves C as it was: the library has no CPU path."""
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from rblas_b200 import level3
    from rblas_b200.error import DeviceError
    from rblas_b200.types import Layout, Transpose

    a, b, c = np.ones(4), np.ones(4), np.full(4, 7.0)
    with pytest.raises(DeviceError):
        level3.gemm(Layout.ColMajor, Transpose.NoTrans, Transpose.NoTrans, 2, 2, 2, 1.0, a, 2, b, 2, 0.0, c, 2)
    assert (c == 7.0).all()
