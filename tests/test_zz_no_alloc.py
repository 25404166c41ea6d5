"""The allocation-free Ozaki DGEMM entry point (rb_dgemm_ozaki_noalloc).

Callers that cannot let a library allocate device memory -- a process that
reserved the whole GPU for its own pool, or a latency-critical path where a
cudaMalloc could block or fail mid-run -- use this entry point instead of
rb_dgemm_dev(..., RB_PREC_OZAKI, ...). It runs the same Ozaki arithmetic, so
it must give the same result on the same inputs, bit for bit. The test calls
it twice in a row through the C ABI (with a smaller second problem, so stale
scratch from the first call would show) and compares each result with the
allocating entry point's: equal, and so also within the normwise tolerance
the GPU tests use (4*k*u_f64). Around a further call it checks that nothing
was allocated: the library's count of device allocations and the device's
free memory do not move. This file is named to be collected last; it also
passes when run on its own.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from rblas_b200 import _lib, level3
from rblas_b200.types import Layout, Precision

pytestmark = pytest.mark.gpu


def _noalloc(layout, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, stream):
    err = _lib.RbError()
    st = _lib.load().rb_dgemm_ozaki_noalloc(int(layout), ta, tb, m, n, k, alpha, C.c_void_p(a), lda,
                                            C.c_void_p(b), ldb, beta, C.c_void_p(c), ldc,
                                            C.c_void_p(stream) if stream else None, C.byref(err))
    return st, err


def _case(torch, layout, ta, tb, m, n, k, seed):
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    ar, ac = (k, m) if ta else (m, k)
    br, bc = (n, k) if tb else (k, n)
    lda = ar if layout == Layout.ColMajor else ac
    ldb = br if layout == Layout.ColMajor else bc
    ldc = m if layout == Layout.ColMajor else n
    A = torch.randn(ar * ac, dtype=torch.float64, device="cuda", generator=g)
    B = torch.randn(br * bc, dtype=torch.float64, device="cuda", generator=g)
    C0 = torch.randn(m * n, dtype=torch.float64, device="cuda", generator=g)
    return A, B, C0, lda, ldb, ldc


@pytest.mark.parametrize("first", [(Layout.ColMajor, 0, 1, 512, 384, 640),
                                   (Layout.RowMajor, 1, 1, 700, 520, 1000)])
def test_noalloc_matches_allocating_entry_point_on_two_calls(first):
    torch = pytest.importorskip("torch")
    stream = torch.cuda.current_stream().cuda_stream
    second = (Layout.RowMajor, 1, 0, 300, 257, 129)
    alpha, beta = 1.5, -0.5
    for i, (layout, ta, tb, m, n, k) in enumerate([first, second]):
        A, B, C0, lda, ldb, ldc = _case(torch, layout, ta, tb, m, n, k, seed=90 + i)
        ref = C0.clone()
        level3.gemm_dev(layout, ta, tb, m, n, k, alpha, A.data_ptr(), lda, B.data_ptr(), ldb, beta,
                        ref.data_ptr(), ldc, np.float64, prec=Precision.Ozaki, stream=stream)
        got = C0.clone()
        st, err = _noalloc(layout, ta, tb, m, n, k, alpha, A.data_ptr(), lda, B.data_ptr(), ldb, beta,
                           got.data_ptr(), ldc, stream)
        assert st == 0, (st, err.code, err.got)
        torch.cuda.synchronize()
        d = (got - ref).double()
        den = abs(alpha) * A.norm().item() * B.norm().item() + abs(beta) * C0.norm().item()
        assert (d.norm().item() / den) <= 4 * k * 2.0 ** -53, f"call {i}: {d.abs().max().item():.3e}"
        assert torch.equal(got, ref), f"call {i}: max diff {d.abs().max().item():.3e}"
    # a third call, after the warm-up above: no device allocation of any kind
    lib = _lib.load()
    layout, ta, tb, m, n, k = first
    A, B, C0, lda, ldb, ldc = _case(torch, layout, ta, tb, m, n, k, seed=97)
    got = C0.clone()
    torch.cuda.synchronize()
    allocs0 = lib.rb_device_alloc_count()
    free0, _ = torch.cuda.mem_get_info()
    st, err = _noalloc(layout, ta, tb, m, n, k, alpha, A.data_ptr(), lda, B.data_ptr(), ldb, beta,
                       got.data_ptr(), ldc, stream)
    assert st == 0, (st, err.code)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert lib.rb_device_alloc_count() == allocs0
    assert free1 == free0, (free0, free1)


def test_noalloc_rejects_problems_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    stream = torch.cuda.current_stream().cuda_stream
    m = n = k = 4096  # needs 8 * 8192 * 4096 bytes of digit planes > 64 MiB
    A = torch.zeros(8, dtype=torch.float64, device="cuda")  # never read: rejected before launch
    C0 = torch.full((8,), 7.0, dtype=torch.float64, device="cuda")
    st, err = _noalloc(Layout.ColMajor, 0, 0, m, n, k, 1.0, A.data_ptr(), m, A.data_ptr(), k, 0.0,
                       C0.data_ptr(), m, stream)
    assert st == 12 and err.code == 12
    assert err.got > err.min_or_need == (64 << 20) + (64 << 10)
    torch.cuda.synchronize()
    assert torch.all(C0 == 7.0)
