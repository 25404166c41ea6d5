"""Host-side failure paths, driven without a GPU fault (rblas's error contract,
src/error.rs:15-39, extended by the device-side statuses of the C ABI).

- An injected allocation failure (rb_debug_inject(RB_INJECT_ALLOC)) makes the
  call that hits it return RB_ERR_ALLOC with its output untouched; the next
  call succeeds.
- A serving batch that finds the device error word set (written from the host
  with rb_debug_inject(RB_INJECT_DEVICE_WORD), as a kernel writes it when a
  bounded wait gives up) fails its requests with RB_ERR_TIMEOUT; the server
  clears the word and the next request is correct. The injected requests have
  k == 0, so the kernels that run while the word is set hold no TMA copy and
  no tensor-core operation in flight when they stop waiting.
- rb_server_cancel cancels a request still waiting for admission.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import oracle
from rblas_b200 import _lib, level3
from rblas_b200.serving import Problem, Server
from rblas_b200.types import Layout, Precision, Transpose

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

RB_ERR_ALLOC, RB_ERR_TIMEOUT, RB_ERR_BUSY, RB_ERR_CANCELLED = 7, 8, 10, 11
RB_INJECT_ALLOC, RB_INJECT_DEVICE_WORD = 1, 2
RB_DEVERR_TIMEOUT = 0x01000000
INJECT_SITE = 0x7E0


def _err():
    return _lib.RbError()


def test_injected_allocation_failure_returns_alloc_and_leaves_c():
    lib = _lib.load()
    m, n, k = 200, 150, 96
    g = torch.Generator(device="cuda")
    g.manual_seed(5)
    A = torch.randn(m * k, dtype=torch.float64, device="cuda", generator=g)
    B = torch.randn(k * n, dtype=torch.float64, device="cuda", generator=g)
    C0 = torch.randn(m * n, dtype=torch.float64, device="cuda", generator=g)
    c = C0.clone()
    torch.cuda.synchronize()
    # the Ozaki form takes its digit planes from the library's scratch pool
    assert lib.rb_debug_inject(RB_INJECT_ALLOC, 0, 1) == 0
    err = _err()
    st = lib.rb_dgemm_dev(1, 0, 0, m, n, k, 1.5, C.c_void_p(A.data_ptr()), m, C.c_void_p(B.data_ptr()), k, -0.5,
                          C.c_void_p(c.data_ptr()), m, int(Precision.Ozaki), None, C.byref(err))
    torch.cuda.synchronize()
    assert st == RB_ERR_ALLOC and err.code == RB_ERR_ALLOC and err.cuda_error == 2  # cudaErrorMemoryAllocation
    assert torch.equal(c, C0)
    # the failure was consumed: the same call now runs and matches the oracle
    err = _err()
    st = lib.rb_dgemm_dev(1, 0, 0, m, n, k, 1.5, C.c_void_p(A.data_ptr()), m, C.c_void_p(B.data_ptr()), k, -0.5,
                          C.c_void_p(c.data_ptr()), m, int(Precision.Ozaki), None, C.byref(err))
    torch.cuda.synchronize()
    assert st == 0, (st, err.code)
    ref = C0.cpu().numpy().copy()
    oracle.gemm(1, 0, 0, m, n, k, 1.5, A.cpu().numpy(), m, B.cpu().numpy(), k, -0.5, ref, m)
    den = 1.5 * float(A.norm()) * float(B.norm()) + 0.5 * float(C0.norm())
    assert np.linalg.norm(c.cpu().numpy() - ref) / den <= 4 * k * 2.0 ** -53


def test_injected_allocation_failure_on_host_call_and_server_create():
    lib = _lib.load()
    rng = np.random.default_rng(8)
    m, n, k = 64, 48, 40
    a = rng.uniform(-1, 1, m * k).astype(np.float32)
    b = rng.uniform(-1, 1, k * n).astype(np.float32)
    c0 = rng.uniform(-1, 1, m * n).astype(np.float32)
    c = c0.copy()
    lib.rb_release_cached_memory()  # so the host call below must allocate its staging buffers
    # a host call first stages its operands into device buffers
    assert lib.rb_debug_inject(RB_INJECT_ALLOC, 0, 1) == 0
    err = _err()
    p = lambda x: C.c_void_p(x.ctypes.data)  # noqa: E731
    st = lib.rb_sgemm(1, 0, 0, m, n, k, 1.0, p(a), m, a.size, p(b), k, b.size, 0.5, p(c), m, c.size, C.byref(err))
    assert st == RB_ERR_ALLOC, (st, err.code)
    assert np.array_equal(c, c0)
    assert lib.rb_debug_inject(RB_INJECT_ALLOC, 0, 0) == 0  # nothing left pending
    level3.gemm(Layout.ColMajor, Transpose.NoTrans, Transpose.NoTrans, m, n, k, 1.0, a, m, b, k, 0.5, c, m)
    ref = c0.copy()
    oracle.gemm(1, 0, 0, m, n, k, 1.0, a, m, b, k, 0.5, ref, m)
    den = float(np.linalg.norm(a.astype(np.float64)) * np.linalg.norm(b.astype(np.float64))) + \
        0.5 * float(np.linalg.norm(c0.astype(np.float64)))
    assert np.linalg.norm(c.astype(np.float64) - ref) / den <= 4 * k * 2.0 ** -24
    # a server's result pool
    assert lib.rb_debug_inject(RB_INJECT_ALLOC, 0, 1) == 0
    h = C.c_void_p()
    assert lib.rb_server_create(1 << 20, 4, 1, C.byref(h)) == RB_ERR_ALLOC
    assert lib.rb_debug_inject(RB_INJECT_ALLOC, 0, 0) == 0
    with Server(budget_bytes=1 << 20, max_batch=4, grouped=True):
        pass


def _k0_problem(dt, m, n, beta, seed):
    """A k == 0 request: D = beta * C0 exactly (no operand is read)."""
    tdt = torch.float32 if dt == np.float32 else torch.float64
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    C0 = torch.randn(m * n, dtype=tdt, device="cuda", generator=g)
    dummy = torch.zeros(16, dtype=tdt, device="cuda")
    p = Problem(dt, Layout.ColMajor, 0, 0, m, n, 0, 1.5, dummy.data_ptr(), m, dummy.data_ptr(), 1, beta,
                C0.data_ptr(), m)
    return p, C0, dummy


def _read(d, m, n, ldd, dt):
    """The server-owned column-major m x n result at device address d, as a
    torch view (m x n)."""
    class _View:
        __cuda_array_interface__ = {"shape": (ldd * n,), "typestr": np.dtype(dt).str, "data": (d, False),
                                    "version": 3}

    torch.cuda.synchronize()
    return torch.as_tensor(_View(), device="cuda").clone().view(n, ldd)[:, :m].T


@pytest.mark.parametrize("grouped", [True, False])
def test_server_reports_device_error_word_then_recovers(grouped):
    lib = _lib.load()
    with Server(budget_bytes=64 << 20, max_batch=8, grouped=grouped) as srv:
        p1, C1, _d1 = _k0_problem(np.float64, 96, 80, -0.5, 11)
        torch.cuda.synchronize()
        assert lib.rb_debug_inject(RB_INJECT_DEVICE_WORD, RB_DEVERR_TIMEOUT | INJECT_SITE, 0) == 0
        rid = srv.submit(p1)
        st, _, _, _ = srv.wait(rid)
        assert st == RB_ERR_TIMEOUT
        assert srv.release(rid) == 0
        # the server cleared the word: the next request runs and is exact
        p2, C2, _d2 = _k0_problem(np.float32, 70, 33, 2.0, 12)
        rid = srv.submit(p2)
        st, d, ldd, _ = srv.wait(rid)
        assert st == 0
        got = _read(d, p2.m, p2.n, ldd, np.float32)
        assert torch.equal(got, (2.0 * C2).view(p2.n, p2.m).T)
        srv.release(rid)
    detail = C.c_uint32(0)
    assert lib.rb_device_error(0, C.byref(detail)) == 0 and detail.value == 0


def test_server_cancel_queued_request():
    # the budget holds one 512 KiB result: the second request waits for memory
    m = n = 256
    with Server(budget_bytes=(m * n * 8) + 4096, max_batch=4, grouped=True) as srv:
        p1, C1, _d1 = _k0_problem(np.float64, m, n, 1.0, 21)
        p2, C2, _d2 = _k0_problem(np.float64, m, n, 1.0, 22)
        r1 = srv.submit(p1)
        st, _, _, _ = srv.wait(r1)
        assert st == 0
        r2 = srv.submit(p2)  # queued behind r1's unreleased result
        st, _, _, _ = srv.wait(r2, timeout_us=20000)
        assert st == RB_ERR_TIMEOUT  # the wait ran out: still queued
        assert srv.cancel(r2) == 0
        st, _, _, _ = srv.wait(r2)
        assert st == RB_ERR_CANCELLED
        assert srv.cancel(r1) == RB_ERR_BUSY  # already ran
        assert srv.cancel(987654321) == 4  # unknown id
        assert srv.release(r2) == 0
        assert srv.release(r1) == 0
        # the freed budget admits the next request at once
        r3 = srv.submit(p2)
        st, d, ldd, _ = srv.wait(r3)
        assert st == 0
        assert torch.equal(_read(d, m, n, ldd, np.float64), C2.view(n, m).T)
        srv.release(r3)
