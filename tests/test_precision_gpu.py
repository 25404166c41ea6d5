"""GPU tests of the split-precision forms (3xBF16 SGEMM and Ozaki INT8-slice
DGEMM on tcgen05), called through the C ABI and checked against the
double-double oracle and against the plain forms on the same inputs.

Tolerances (stated here, used below):
  * OZAKI  normwise error vs the double-double oracle <= 4*k*u_f64 (the plain
    form's parity bound) and <= 2x the plain DGEMM's own error + 2^-52.
  * BF16X3 normwise error vs the double-double oracle <= 2^-15 (three bf16
    products keep ~16 significand bits per product; the dropped lo*lo term
    and split residuals are ~2^-17 relative).
  * BF16X6 (three planes, six products) normwise error <= 4*k*u_f32, the
    plain SGEMM parity bound; at the SGEMM configuration sizes (8192^3 and
    65536x128x8192, uniform and log-uniform inputs) also <= 2x the plain
    form's own error.
  * 3xBF16 at those sizes: <= 6x the plain form's error. Its hi + lo split
    keeps ~17 significand bits per operand, so it cannot reach 2x plain
    there (measured 2.3-5.6x); the bound guards against regressions.
"""
from __future__ import annotations

import json
import os

import numpy as np
import pytest

import oracle
import rblas_b200 as rb
from rblas_b200 import level3
from rblas_b200.types import Layout, Precision
from tests.util import Problem

pytestmark = pytest.mark.gpu

BF16X3_TOL = 2.0 ** -15


def run(p: Problem, prec):
    c = p.fresh_c()
    level3.gemm(p.layout, p.ta, p.tb, p.m, p.n, p.k, p.alpha, p.a, p.lda, p.b, p.ldb, p.beta, c,
                p.ldc, prec=prec)
    return c


SHAPES = [(1, 1, 1), (17, 13, 19), (129, 257, 33), (300, 520, 1000), (256, 256, 4096)]


@pytest.mark.parametrize("layout", [Layout.ColMajor, Layout.RowMajor])
@pytest.mark.parametrize("ta", [0, 1])
@pytest.mark.parametrize("tb", [0, 1])
def test_ozaki_accuracy_all_transposes(layout, ta, tb):
    for i, (m, n, k) in enumerate(SHAPES):
        p = Problem(layout, ta, tb, m, n, k, np.float64, alpha=1.5, beta=-0.5, seed=200 + i,
                    dist="normal")
        c = run(p, Precision.Ozaki)
        err = p.normwise_vs_dd(c)
        plain = p.normwise_vs_dd(run(p, Precision.Plain))
        assert err <= p.tol(), f"{(m, n, k)} ozaki {err:.3e} > {p.tol():.3e}"
        assert err <= 2 * plain + 2.0 ** -52, f"{(m, n, k)} ozaki {err:.3e} vs plain {plain:.3e}"
    assert rb.device_error()[0] == 0


@pytest.mark.parametrize("layout", [Layout.ColMajor, Layout.RowMajor])
@pytest.mark.parametrize("ta", [0, 1])
@pytest.mark.parametrize("tb", [0, 1])
def test_bf16x3_accuracy_all_transposes(layout, ta, tb):
    for i, (m, n, k) in enumerate(SHAPES):
        p = Problem(layout, ta, tb, m, n, k, np.float32, alpha=1.0, beta=1.0, seed=300 + i)
        c = run(p, Precision.Bf16x3)
        err = p.normwise_vs_dd(c)
        assert err <= BF16X3_TOL, f"{(m, n, k)} bf16x3 {err:.3e}"
    assert rb.device_error()[0] == 0


@pytest.mark.parametrize("layout", [Layout.ColMajor, Layout.RowMajor])
@pytest.mark.parametrize("ta", [0, 1])
@pytest.mark.parametrize("tb", [0, 1])
def test_bf16x6_accuracy_all_transposes(layout, ta, tb):
    for i, (m, n, k) in enumerate(SHAPES):
        p = Problem(layout, ta, tb, m, n, k, np.float32, alpha=1.0, beta=1.0, seed=400 + i)
        c = run(p, Precision.Bf16x6)
        err = p.normwise_vs_dd(c)
        assert err <= p.tol(), f"{(m, n, k)} bf16x6 {err:.3e}"
        assert err <= p.normwise_vs_dd(run(p, Precision.Bf16x3)) + 1e-12
    assert rb.device_error()[0] == 0


def test_ozaki_wide_exponent_stress():
    """Entries sign*2^e, e ~ U{-30..30}: per-row scaling still meets the bound."""
    for ta, tb in [(0, 0), (1, 1)]:
        p = Problem(Layout.RowMajor, ta, tb, 192, 160, 700, np.float64, alpha=1.5, beta=-0.5,
                    seed=21, dist="pow2")
        err = p.normwise_vs_dd(run(p, Precision.Ozaki))
        plain = p.normwise_vs_dd(run(p, Precision.Plain))
        assert err <= 2 * plain + 2.0 ** -52, (err, plain)


def test_bf16x3_loguniform_inputs():
    p = Problem(Layout.ColMajor, 0, 0, 256, 256, 2048, np.float32, alpha=1.0, beta=1.0, seed=22,
                dist="loguniform")
    err = p.normwise_vs_dd(run(p, Precision.Bf16x3))
    assert err <= BF16X3_TOL, err


def test_ozaki_zero_rows_and_columns():
    p = Problem(Layout.ColMajor, 0, 0, 70, 60, 90, np.float64, alpha=2.0, beta=0.5, seed=23,
                dist="normal")
    A = oracle.stored_2d(p.a, 70, 90, p.lda, 1)
    A[5, :] = 0.0
    p.A[5, :] = 0.0
    B = oracle.stored_2d(p.b, 90, 60, p.ldb, 1)
    B[:, 7] = 0.0
    p.B[:, 7] = 0.0
    c = run(p, Precision.Ozaki)
    assert p.normwise_vs_dd(c) <= p.tol()
    # row 5 and column 7 are exactly beta*C0
    R = p.result(c)
    assert np.array_equal(R[5, :], 0.5 * p.C0[5, :])
    assert np.array_equal(R[:, 7], 0.5 * p.C0[:, 7])


@pytest.mark.parametrize("prec,dtype", [(Precision.Ozaki, np.float64), (Precision.Bf16x3, np.float32),
                                        (Precision.Bf16x6, np.float32)])
def test_beta_zero_nan_c_and_alpha_zero(prec, dtype):
    p = Problem(Layout.ColMajor, 0, 1, 40, 33, 50, dtype, alpha=1.0, beta=0.0, seed=24, c0_nan=True)
    c = run(p, prec)
    assert not np.any(np.isnan(p.result(c)))
    p = Problem(Layout.ColMajor, 0, 0, 40, 33, 50, dtype, alpha=0.0, beta=-2.0, seed=25)
    c = run(p, prec)
    assert np.array_equal(p.result(c), p.result(p.reference_restatement()))


def test_ozaki_slice_count_controls_accuracy():
    p = Problem(Layout.ColMajor, 0, 0, 128, 256, 512, np.float64, seed=26, dist="normal")
    errs = {}
    try:
        for s in (4, 6, 8):
            assert rb._lib.load().rb_set_ozaki_slices(s) == 0
            errs[s] = p.normwise_vs_dd(run(p, Precision.Ozaki))
    finally:
        rb._lib.load().rb_set_ozaki_slices(8)
    assert errs[4] > errs[6] > errs[8]


def test_unsupported_pairings_are_rejected():
    p = Problem(Layout.ColMajor, 0, 0, 8, 8, 8, np.float32, seed=27)
    with pytest.raises(rb.DeviceError) as ei:
        run(p, Precision.Ozaki)
    assert ei.value.code == 5
    p = Problem(Layout.ColMajor, 0, 0, 8, 8, 8, np.float64, seed=27)
    with pytest.raises(rb.DeviceError):
        run(p, Precision.Bf16x3)


def _report_path():
    """Where to write the error report: the file named by RB_PRECISION_REPORT, if set."""
    return os.environ.get("RB_PRECISION_REPORT") or None


def test_config_sizes_error_report():
    """Errors at the configuration sizes (row-sampled double-double oracle):
    DGEMM 4096^3 row-major all four transposes (normal and 2^e sets), and
    SGEMM 8192^3 / 65536x128x8192 col-major beta=1 (uniform and log-uniform).
    Asserts the targets; writes the numbers to the file named by
    RB_PRECISION_REPORT when that is set."""
    rng = np.random.default_rng(99)
    report = {}
    for dist in ("normal", "pow2"):
        for ta, tb in [(0, 0), (1, 0), (0, 1), (1, 1)]:
            p = Problem(Layout.RowMajor, ta, tb, 4096, 4096, 4096, np.float64, alpha=1.5, beta=-0.5,
                        seed=31, dist=dist)
            rows = np.sort(rng.choice(4096, 64, replace=False))
            e_pl = p.normwise_vs_dd(run(p, Precision.Plain), rows=rows)
            e_oz = p.normwise_vs_dd(run(p, Precision.Ozaki), rows=rows)
            report[f"dgemm_4096_{dist}_{'NT'[ta]}{'NT'[tb]}"] = {"plain": e_pl, "ozaki": e_oz}
            assert e_oz <= 2 * e_pl + 2.0 ** -52
    for (m, n, k) in [(8192, 8192, 8192), (65536, 128, 8192)]:
        for dist in ("uniform", "loguniform"):
            p = Problem(Layout.ColMajor, 0, 0, m, n, k, np.float32, alpha=1.0, beta=1.0, seed=32,
                        dist=dist)
            rows = np.sort(rng.choice(m, 32, replace=False))
            e_pl = p.normwise_vs_dd(run(p, Precision.Plain), rows=rows)
            e_b3 = p.normwise_vs_dd(run(p, Precision.Bf16x3), rows=rows)
            e_b6 = p.normwise_vs_dd(run(p, Precision.Bf16x6), rows=rows)
            report[f"sgemm_{m}x{n}x{k}_{dist}"] = {"plain": e_pl, "bf16x3": e_b3, "bf16x6": e_b6,
                                                  "ratio_x3": e_b3 / e_pl if e_pl else None,
                                                  "ratio_x6": e_b6 / e_pl if e_pl else None}
    path = _report_path()
    if path:
        with open(path, "w") as f:
            json.dump(report, f, indent=1)
    print(json.dumps(report, indent=1))
    for key, r in report.items():
        if key.startswith("sgemm_"):
            assert r["bf16x6"] <= 2 * r["plain"], (key, r)
            assert r["bf16x3"] <= 6 * r["plain"], (key, r)


@pytest.mark.parametrize("layout,ta,tb,m,n,k", [(Layout.ColMajor, 0, 0, 300, 257, 513),
                                                 (Layout.RowMajor, 1, 1, 1000, 900, 700),
                                                 (Layout.ColMajor, 1, 0, 64, 64, 4096),
                                                 (Layout.ColMajor, 0, 0, 2560, 2048, 512),
                                                 (Layout.RowMajor, 1, 0, 3200, 2048, 1024)])
def test_ozaki_unit_parallel_matches_fused_epilogue_exactly(layout, ta, tb, m, n, k):
    """Tiles that would leave SMs idle -- all of them when there are fewer
    tiles than SMs (the first three shapes), the partial last wave otherwise
    (2560 x 2048: one full wave of 148 tiles and 12 split; 3200 x 2048: 52
    split, dealt over two snake passes) -- run one diagonal-pair unit per work
    item and fold the units' exact terms in unit order afterwards; that is the
    fused epilogue's arithmetic, so the result equals the fused path's (run
    here through the allocation-free entry point, which always fuses) bit
    for bit -- including a zero row, a zero column and beta = 0 with NaN C."""
    import ctypes as C
    torch = pytest.importorskip("torch")
    from rblas_b200 import _lib
    g = torch.Generator(device="cuda")
    g.manual_seed(m + n)
    ar, ac = (k, m) if ta else (m, k)
    br, bc = (n, k) if tb else (k, n)
    lda = ar if layout == Layout.ColMajor else ac
    ldb = br if layout == Layout.ColMajor else bc
    ldc = m if layout == Layout.ColMajor else n
    A = torch.randn(ar * ac, dtype=torch.float64, device="cuda", generator=g)
    B = torch.randn(br * bc, dtype=torch.float64, device="cuda", generator=g)
    # a zero row of op(A): row 3 of A (stored rows when NoTrans col-major)
    if layout == Layout.ColMajor and not ta:
        A.view(ac, ar)[:, 3] = 0.0
    for beta, fill in ((-0.5, None), (0.0, float("nan"))):
        C0 = torch.randn(m * n, dtype=torch.float64, device="cuda", generator=g)
        if fill is not None:
            C0.fill_(fill)
        got, ref = C0.clone(), C0.clone()
        level3.gemm_dev(layout, ta, tb, m, n, k, 1.25, A.data_ptr(), lda, B.data_ptr(), ldb, beta, got.data_ptr(),
                        ldc, np.float64, prec=Precision.Ozaki)
        err = _lib.RbError()
        st = _lib.load().rb_dgemm_ozaki_noalloc(int(layout), ta, tb, m, n, k, 1.25, C.c_void_p(A.data_ptr()), lda,
                                                C.c_void_p(B.data_ptr()), ldb, beta, C.c_void_p(ref.data_ptr()), ldc,
                                                None, C.byref(err))
        assert st == 0
        torch.cuda.synchronize()
        assert torch.equal(got, ref) or torch.allclose(got, ref, rtol=0, atol=0, equal_nan=True)


@pytest.mark.parametrize("prec", [Precision.Bf16x3, Precision.Bf16x6])
@pytest.mark.parametrize("m,n,k,beta", [(1000, 200, 777, -0.5), (300, 128, 64, 0.0), (129, 1, 4096, 1.0),
                                        (65536, 128, 8192, 1.0)])
def test_bf16_split_in_gemm_matches_two_pass_exactly(m, n, k, beta, prec):
    """An A with contiguous rows (ColMajor NoTrans) and at most two 128-wide
    column tiles runs the BF16-split form with A split inside the GEMM; the
    same product with A stored transposed (Trans) takes the split pass and
    the two-pass kernel. Same planes, same products in the same order, same
    accumulators and promotions: equal bit for bit. Ragged rows, columns and
    K, a partial last accumulation unit, beta = 0 with NaN C0, and the
    tall-skinny 65536 x 128 x 8192 configuration."""
    torch = pytest.importorskip("torch")
    g = torch.Generator(device="cuda")
    g.manual_seed(m + n + k)
    A = torch.rand(m * k, dtype=torch.float32, device="cuda", generator=g) * 2 - 1  # m x k, lda = m
    At = A.view(k, m).t().contiguous().view(-1)  # the same matrix stored k x m (lda = k)
    B = torch.rand(k * n, dtype=torch.float32, device="cuda", generator=g) * 2 - 1
    C0 = torch.rand(m * n, dtype=torch.float32, device="cuda", generator=g) * 2 - 1
    if beta == 0.0:
        C0.fill_(float("nan"))
    fused, two_pass = C0.clone(), C0.clone()
    level3.gemm_dev(Layout.ColMajor, 0, 0, m, n, k, 1.25, A.data_ptr(), m, B.data_ptr(), k, beta, fused.data_ptr(),
                    m, np.float32, prec=prec)
    level3.gemm_dev(Layout.ColMajor, 1, 0, m, n, k, 1.25, At.data_ptr(), k, B.data_ptr(), k, beta,
                    two_pass.data_ptr(), m, np.float32, prec=prec)
    torch.cuda.synchronize()
    assert not torch.isnan(fused).any()
    assert torch.equal(fused, two_pass)
    assert rb.device_error()[0] == 0
