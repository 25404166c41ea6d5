"""GPU parity tests of the plain GEMM forms (true-FP32 SGEMM, FP64 DGEMM),
called through the C ABI (rblas_b200.level3 -> librblas_b200.so) and checked
against the oracle: the reference's own test assertions (golden cases), the
CPU restatement of rblas's gemm on the same seeded inputs within the stated
normwise tolerance 4*k*u, and the double-double accuracy oracle."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import oracle
import rblas_b200 as rb
from rblas_b200 import level3
from rblas_b200.types import Layout, Transpose
from tests.golden_runner import load_cases, run_case
from tests.util import Problem

pytestmark = pytest.mark.gpu

CASES = load_cases()
GEMM_CASES = sorted(n for n, (m, _) in CASES.items() if m["op"] == "gemm")


class GpuBackend:
    def gemm(self, layout, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
        level3.gemm(layout, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)


@pytest.mark.parametrize("name", GEMM_CASES)
def test_reference_test_cases_on_gpu(name):
    meta, data = CASES[name]
    ok, detail = run_case(GpuBackend(), meta, data)
    assert ok, f"{name} ({meta['ref']}): {detail}"


def _gpu_gemm(p: Problem):
    c = p.fresh_c()
    level3.gemm(p.layout, p.ta, p.tb, p.m, p.n, p.k, p.alpha, p.a, p.lda, p.b, p.ldb, p.beta, c,
                p.ldc)
    return c


SHAPES = [(1, 1, 1), (17, 13, 19), (129, 257, 33), (300, 200, 1000), (64, 5000, 48), (7, 300, 517)]


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("layout", [Layout.ColMajor, Layout.RowMajor])
@pytest.mark.parametrize("ta", [0, 1])
@pytest.mark.parametrize("tb", [0, 1])
def test_parity_all_layouts_and_transposes(dtype, layout, ta, tb):
    for i, (m, n, k) in enumerate(SHAPES):
        p = Problem(layout, ta, tb, m, n, k, dtype, alpha=1.5, beta=-0.5, seed=100 + i)
        c = _gpu_gemm(p)
        ref = p.reference_restatement()
        err = p.normwise(c, ref)
        assert err <= p.tol(), f"{(m, n, k)} normwise vs restatement {err:.3e} > {p.tol():.3e}"
        assert p.normwise_vs_dd(c) <= p.tol()


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_padded_leading_dims_preserve_padding(dtype):
    p = Problem(Layout.ColMajor, 0, 1, 70, 45, 33, dtype, alpha=0.75, beta=2.0, pad=5, seed=7)
    c = _gpu_gemm(p)
    # padding (NaN) slots of C are untouched; the matrix part matches
    full = np.ones(c.size, bool)
    view = oracle.stored_2d(full, p.m, p.n, p.ldc, 1)
    view[...] = False
    assert np.all(np.isnan(c[full]))
    assert p.normwise(c, p.reference_restatement()) <= p.tol()


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_beta_zero_ignores_nan_in_c(dtype):
    """apply_beta (src/kernel/gemm.rs:322-338): beta == 0 never reads C."""
    p = Problem(Layout.ColMajor, 0, 0, 33, 21, 40, dtype, alpha=1.0, beta=0.0, seed=8, c0_nan=True)
    c = _gpu_gemm(p)
    assert not np.any(np.isnan(p.result(c)))
    assert p.normwise(c, p.reference_restatement()) <= p.tol()


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_alpha_zero_and_k_zero_scale_c_only(dtype):
    for beta in (0.0, 1.0, -3.0):
        p = Problem(Layout.RowMajor, 1, 0, 9, 11, 6, dtype, alpha=0.0, beta=beta, seed=9)
        c = _gpu_gemm(p)
        ref = p.reference_restatement()
        assert np.array_equal(p.result(c), p.result(ref))
    p = Problem(Layout.ColMajor, 0, 0, 9, 11, 0, dtype, alpha=1.0, beta=0.5, seed=10)
    c = _gpu_gemm(p)
    assert np.array_equal(p.result(c), p.result(p.reference_restatement()))


@pytest.mark.parametrize("layout", [Layout.ColMajor, Layout.RowMajor])
@pytest.mark.parametrize("ta", [0, 1])
@pytest.mark.parametrize("tb", [0, 1])
def test_narrow_f32_tile_parity(layout, ta, tb):
    """f32 shapes whose 128 x 128 tiles leave SMs idle while 128 x 64 tiles
    fill them (the narrow tile, no split-K), ragged edges included."""
    for i, (m, n, k) in enumerate([(1000, 1000, 777), (900, 1100, 300), (1024, 960, 64)]):
        p = Problem(layout, ta, tb, m, n, k, np.float32, alpha=1.5, beta=-0.5, seed=300 + i)
        c = _gpu_gemm(p)
        ref = p.reference_restatement()
        err = p.normwise(c, ref)
        assert err <= p.tol(), f"{(m, n, k)} normwise vs restatement {err:.3e} > {p.tol():.3e}"
        rows = np.sort(np.random.default_rng(7 + i).choice(p.m, 32, replace=False))
        assert p.normwise_vs_dd(c, rows=rows) <= p.tol()


def test_sgemm_1024_colmajor_nn_matches_rblas():
    """Plain SGEMM, f32, col-major NN, 1024^3, alpha=1, beta=0, A/B from the
    reference tests' LCG (seed 0x12345678): within 4*k*u_f32 normwise of the
    restatement of rblas's own gemm on identical inputs."""
    m = n = k = 1024
    vals, _ = oracle.lcg_f32(0x12345678, m * k + k * n, 0)
    a, b = vals[:m * k].copy(), vals[m * k:].copy()
    c = np.zeros(m * n, np.float32)
    level3.gemm(Layout.ColMajor, Transpose.NoTrans, Transpose.NoTrans, m, n, k, 1.0, a, m, b, k,
                0.0, c, m)
    ref = np.zeros(m * n, np.float32)
    oracle.gemm(1, 0, 0, m, n, k, 1.0, a, m, b, k, 0.0, ref, m)
    d = (c.astype(np.float64) - ref).reshape(-1)
    den = np.linalg.norm(a.astype(np.float64)) * np.linalg.norm(b.astype(np.float64))
    err = np.sqrt(np.sum(d * d)) / den
    assert err <= 4 * k * 2.0 ** -24, err


def test_device_pointer_path_with_unaligned_leading_dim():
    """lda*4 bytes not a multiple of 16 and an odd base offset: the device
    entry point repacks for TMA and still computes the right product."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(11)
    m, n, k = 61, 37, 45
    lda, ldb, ldc = 63, 47, 65
    A = torch.tensor(rng.uniform(-1, 1, lda * k + 1), dtype=torch.float32, device="cuda")
    B = torch.tensor(rng.uniform(-1, 1, ldb * n), dtype=torch.float32, device="cuda")
    Cd = torch.zeros(ldc * n, dtype=torch.float32, device="cuda")
    a_off = A[1:]  # 4-byte misaligned base
    level3.gemm_dev(Layout.ColMajor, 0, 0, m, n, k, 1.0, a_off.data_ptr(), lda, B.data_ptr(), ldb,
                    0.0, Cd.data_ptr(), ldc, np.float32,
                    stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    a_h = a_off.cpu().numpy()
    b_h = B.cpu().numpy()
    c_h = Cd.cpu().numpy()
    ref = np.zeros(ldc * n, np.float32)
    oracle.gemm(1, 0, 0, m, n, k, 1.0, a_h, lda, b_h, ldb, 0.0, ref, ldc)
    got = oracle.stored_2d(c_h, m, n, ldc, 1)
    want = oracle.stored_2d(ref, m, n, ldc, 1)
    assert np.max(np.abs(got - want)) < 1e-4
    assert rb.device_error()[0] == 0


def test_launch_counter_advances():
    before = rb.launch_count()
    p = Problem(Layout.ColMajor, 0, 0, 64, 64, 64, np.float32, seed=12)
    _gpu_gemm(p)
    assert rb.launch_count() > before


@pytest.mark.parametrize("dtype,prec", [(np.float64, 0), (np.float64, 2), (np.float32, 0), (np.float32, 3)])
@pytest.mark.parametrize("layout,ta,tb,m,n,k", [(Layout.ColMajor, 0, 0, 2600, 1300, 2600),
                                                 (Layout.RowMajor, 1, 1, 2400, 1536, 2600),
                                                 (Layout.ColMajor, 1, 0, 3072, 2304, 1400)])
def test_pipelined_host_call_matches_device_call_exactly(dtype, prec, layout, ta, tb, m, n, k):
    """Host-slice calls of at least 64 MB run as column panels on several
    streams; every element is computed as in one whole call, so the result
    equals the device-pointer call on the same data bit for bit (ragged last
    panel, transposes, both layouts, plain and precision forms)."""
    torch = pytest.importorskip("torch")
    from rblas_b200.types import Precision
    rng = np.random.default_rng(120 + m)
    ar, ac = (k, m) if ta else (m, k)
    br, bc = (n, k) if tb else (k, n)
    contig = (lambda r, c: r) if layout == Layout.ColMajor else (lambda r, c: c)
    lda, ldb, ldc = contig(ar, ac), contig(br, bc), contig(m, n)
    a = rng.standard_normal(ar * ac).astype(dtype)
    b = rng.standard_normal(br * bc).astype(dtype)
    c0 = rng.standard_normal(m * n).astype(dtype)
    assert (a.nbytes + b.nbytes + 2 * c0.nbytes) >= 64 << 20
    host = c0.copy()
    level3.gemm(layout, ta, tb, m, n, k, 1.25, a, lda, b, ldb, -0.5, host, ldc, prec=Precision(prec))
    tdt = torch.float32 if dtype == np.float32 else torch.float64
    A, B, Cd = (torch.tensor(x, dtype=tdt, device="cuda") for x in (a, b, c0))
    level3.gemm_dev(layout, ta, tb, m, n, k, 1.25, A.data_ptr(), lda, B.data_ptr(), ldb, -0.5, Cd.data_ptr(), ldc,
                    dtype, prec=Precision(prec))
    torch.cuda.synchronize()
    assert np.array_equal(host, Cd.cpu().numpy())


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_long_k_results_repeat_bit_for_bit(dtype, ta, tb):
    """Each compute warp fences its shared-memory reads before releasing a
    pipeline stage. Without that fence the producer's next TMA write could
    land under reads still in flight, which showed up as whole 16-row
    fragment blocks wrong, differently from call to call, once K spanned
    many stages. Three calls on 512^3 must agree bit for bit and with the
    restatement."""
    torch = pytest.importorskip("torch")
    m = n = k = 512
    tdt = torch.float32 if dtype == np.float32 else torch.float64
    g = torch.Generator(device="cuda")
    g.manual_seed(31 + 2 * ta + tb)
    A = torch.randn(m * k, dtype=tdt, device="cuda", generator=g)
    B = torch.randn(k * n, dtype=tdt, device="cuda", generator=g)
    lda, ldb = (k if ta else m), (n if tb else k)
    outs = []
    for _ in range(3):
        C = torch.zeros(m * n, dtype=tdt, device="cuda")
        level3.gemm_dev(Layout.ColMajor, ta, tb, m, n, k, 1.0, A.data_ptr(), lda, B.data_ptr(), ldb, 0.0,
                        C.data_ptr(), m, dtype)
        torch.cuda.synchronize()
        outs.append(C.cpu().numpy())
    assert np.array_equal(outs[0], outs[1]) and np.array_equal(outs[0], outs[2])
    a = A.cpu().numpy().astype(np.float64).reshape((k, m) if not ta else (m, k)).T  # column-major views
    b = B.cpu().numpy().astype(np.float64).reshape((n, k) if not tb else (k, n)).T
    opa = a.T if ta else a
    opb = b.T if tb else b
    ref = opa @ opb
    got = outs[0].astype(np.float64).reshape(n, m).T
    u = 2.0 ** -24 if dtype == np.float32 else 2.0 ** -53
    err = np.linalg.norm(got - ref) / (np.linalg.norm(opa) * np.linalg.norm(opb))
    assert err <= 4 * k * u, err
