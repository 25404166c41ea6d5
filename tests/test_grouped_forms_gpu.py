"""The grouped precision-form launches: rb_gemm_grouped_ozaki_dev (many f64
GEMMs -- each one call of rblas's level3::gemm::<f64>, src/level3.rs:32-62 --
in the Ozaki INT8 form with one exponent pass, one slice pass and one
persistent tensor-core kernel for the whole batch) and
rb_gemm_grouped_bf16_dev (many f32 GEMMs in 3xBF16 or BF16X6 with one split
pass and one persistent kernel).

Every tile runs the single-problem kernel's epilogue, in the same order of
operations, so each result must equal that problem's own rb_?gemm_dev call
in the same form bit for bit (NaN where it has NaN), and so also meet the
tolerances the other tests state (Ozaki: 4*k*u_f64 normwise against the
oracle, checked here on a few problems).
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from rblas_b200 import level3
from rblas_b200.serving import Problem, grouped_gemm_bf16, grouped_gemm_ozaki
from rblas_b200.types import Layout, Precision

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _problem(rng, layout, ta, tb, m, n, k, alpha, beta, pad=0, c_fill=None, dtype=torch.float64):
    ar, ac = (k, m) if ta else (m, k)
    br, bc = (n, k) if tb else (k, n)
    contig = (lambda r, c: r) if layout == Layout.ColMajor else (lambda r, c: c)
    lda, ldb, ldc = max(contig(ar, ac), 1) + pad, max(contig(br, bc), 1) + pad, max(contig(m, n), 1)
    A = torch.tensor(rng.standard_normal(max(lda * (ac if layout == Layout.ColMajor else ar), 1)),
                     dtype=dtype, device="cuda")
    B = torch.tensor(rng.standard_normal(max(ldb * (bc if layout == Layout.ColMajor else br), 1)),
                     dtype=dtype, device="cuda")
    C0 = torch.tensor(rng.standard_normal(max(m * n, 1)), dtype=dtype, device="cuda")
    if c_fill is not None:
        C0.fill_(c_fill)
    return dict(layout=layout, ta=ta, tb=tb, m=m, n=n, k=k, alpha=alpha, beta=beta, A=A, B=B, C0=C0,
                lda=lda, ldb=ldb, ldc=ldc, dtype=np.float64 if dtype == torch.float64 else np.float32)


def _mix(rng, dtype=torch.float64):
    out = []
    for _ in range(36):
        layout = [Layout.RowMajor, Layout.ColMajor][rng.integers(2)]
        ta, tb = int(rng.integers(3)), int(rng.integers(3))
        m, n, k = (int(np.exp(rng.uniform(0, np.log(900)))) for _ in range(3))
        out.append(_problem(rng, layout, ta, tb, m, n, k, float(rng.uniform(-2, 2)), float(rng.uniform(-2, 2)),
                            dtype=dtype))
    # a few large ones (several tiles each, K of several 128-wide steps)
    out.append(_problem(rng, Layout.RowMajor, 1, 0, 1500, 1200, 900, 1.5, -0.5, dtype=dtype))
    out.append(_problem(rng, Layout.ColMajor, 0, 1, 700, 2100, 1300, -0.75, 1.0, dtype=dtype))
    out.append(_problem(rng, Layout.ColMajor, 2, 2, 257, 511, 2049, 0.5, 0.0, dtype=dtype))
    # edge cases: k == 0, alpha == 0, beta == 0 with NaN C, an empty C, padded leading dims
    out.append(_problem(rng, Layout.ColMajor, 0, 0, 33, 17, 0, 1.5, -0.5, dtype=dtype))
    out.append(_problem(rng, Layout.RowMajor, 1, 0, 40, 21, 13, 0.0, 2.0, dtype=dtype))
    out.append(_problem(rng, Layout.ColMajor, 0, 1, 64, 48, 96, 1.25, 0.0, c_fill=float("nan"), dtype=dtype))
    out.append(_problem(rng, Layout.ColMajor, 0, 0, 0, 5, 7, 1.0, 1.0, dtype=dtype))
    out.append(_problem(rng, Layout.RowMajor, 0, 1, 150, 130, 170, -1.0, 0.75, pad=3, dtype=dtype))
    return out


def _as_problem(d, c):
    return Problem(d["dtype"], d["layout"], d["ta"], d["tb"], d["m"], d["n"], d["k"], d["alpha"], d["A"].data_ptr(),
                   d["lda"], d["B"].data_ptr(), d["ldb"], d["beta"], c.data_ptr(), d["ldc"])


def _same(g, ref):
    return torch.equal(g, ref) or bool(torch.all((g == ref) | (torch.isnan(g) & torch.isnan(ref))))


def test_grouped_ozaki_equals_single_ozaki_calls_bit_for_bit():
    rng = np.random.default_rng(70)
    mix = _mix(rng)
    got = [d["C0"].clone() for d in mix]
    grouped_gemm_ozaki([_as_problem(d, c) for d, c in zip(mix, got)])
    torch.cuda.synchronize()
    for i, (d, g) in enumerate(zip(mix, got)):
        ref = d["C0"].clone()
        level3.gemm_dev(d["layout"], d["ta"], d["tb"], d["m"], d["n"], d["k"], d["alpha"], d["A"].data_ptr(),
                        d["lda"], d["B"].data_ptr(), d["ldb"], d["beta"], ref.data_ptr(), d["ldc"], np.float64,
                        prec=Precision.Ozaki)
        torch.cuda.synchronize()
        assert _same(g, ref), (i, d["layout"], d["ta"], d["tb"], d["m"], d["n"], d["k"], (g - ref).abs().max().item())
    # beta == 0 never reads C: the NaN-filled case comes out finite
    assert bool(torch.isfinite(got[-3]).all())


def test_grouped_ozaki_meets_the_oracle_bound():
    rng = np.random.default_rng(71)
    mix = [_problem(rng, Layout.RowMajor, 0, 0, 300, 260, 700, 1.5, -0.5),
           _problem(rng, Layout.ColMajor, 1, 1, 513, 129, 1025, -0.5, 1.0)]
    got = [d["C0"].clone() for d in mix]
    grouped_gemm_ozaki([_as_problem(d, c) for d, c in zip(mix, got)])
    torch.cuda.synchronize()
    for d, g in zip(mix, got):
        layout = int(d["layout"])
        a, b, c0 = (t.cpu().numpy() for t in (d["A"], d["B"], d["C0"]))
        hi, lo = oracle.dd_gemm(layout, d["ta"], d["tb"], d["m"], d["n"], d["k"], d["alpha"], a, d["lda"], b,
                                d["ldb"], d["beta"], c0, d["ldc"])
        r = oracle.stored_2d(g.cpu().numpy(), d["m"], d["n"], d["ldc"], layout)
        diff = (r - hi) - lo
        A = oracle.stored_2d(a, *((d["k"], d["m"]) if d["ta"] else (d["m"], d["k"])), d["lda"], layout)
        B = oracle.stored_2d(b, *((d["n"], d["k"]) if d["tb"] else (d["k"], d["n"])), d["ldb"], layout)
        den = abs(d["alpha"]) * np.linalg.norm(A) * np.linalg.norm(B) + abs(d["beta"]) * np.linalg.norm(c0)
        assert np.linalg.norm(diff) / den <= 4 * d["k"] * 2.0 ** -53


@pytest.mark.parametrize("prec", [Precision.Bf16x3, Precision.Bf16x6])
def test_grouped_bf16_equals_single_calls_bit_for_bit(prec):
    rng = np.random.default_rng(72 + int(prec))
    mix = _mix(rng, dtype=torch.float32)
    got = [d["C0"].clone() for d in mix]
    grouped_gemm_bf16([_as_problem(d, c) for d, c in zip(mix, got)], prec)
    torch.cuda.synchronize()
    for i, (d, g) in enumerate(zip(mix, got)):
        ref = d["C0"].clone()
        level3.gemm_dev(d["layout"], d["ta"], d["tb"], d["m"], d["n"], d["k"], d["alpha"], d["A"].data_ptr(),
                        d["lda"], d["B"].data_ptr(), d["ldb"], d["beta"], ref.data_ptr(), d["ldc"], np.float32,
                        prec=prec)
        torch.cuda.synchronize()
        assert _same(g, ref), (i, d["layout"], d["ta"], d["tb"], d["m"], d["n"], d["k"], (g - ref).abs().max().item())
    assert bool(torch.isfinite(got[-3]).all())  # beta == 0 never reads the NaN-filled C
