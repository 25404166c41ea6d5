"""Shared helpers for the parity tests: seeded problem generation in rblas's
buffer conventions and the normwise parity metric."""
from __future__ import annotations

import numpy as np

import oracle


def stored_shape(layout, trans, rows, cols):
    """(stored_rows, stored_cols) of op(X) = rows x cols under `trans`."""
    return (cols, rows) if trans else (rows, cols)


def make_buffer(rng, layout, rows, cols, ld, dtype, dist="uniform"):
    """A flat BLAS buffer holding a rows x cols matrix with leading dim ld.
    Padding slots hold NaN so any out-of-matrix read shows up."""
    if layout == 1:
        size = (cols - 1) * ld + rows if rows and cols else 0
    else:
        size = (rows - 1) * ld + cols if rows and cols else 0
    buf = np.full(size, np.nan, dtype=dtype)
    mat = sample(rng, (rows, cols), dtype, dist)
    if size:
        view = oracle.stored_2d(buf, rows, cols, ld, layout)
        view[...] = mat
    return buf, mat


def sample(rng, shape, dtype, dist="uniform"):
    if dist == "uniform" and np.dtype(dtype) == np.float32:
        return (rng.random(shape, dtype=np.float32) * np.float32(2.0) - np.float32(1.0))
    if dist == "uniform":
        x = rng.uniform(-1.0, 1.0, shape)
    elif dist == "normal":
        x = rng.standard_normal(shape)
    elif dist == "pow2":  # sign * 2^e, e ~ U{-30..30}
        x = np.sign(rng.uniform(-1, 1, shape)) * np.exp2(rng.integers(-30, 31, shape))
    elif dist == "loguniform":  # |x| in [2^-20, 2^20], random sign
        x = np.sign(rng.uniform(-1, 1, shape)) * np.exp2(rng.uniform(-20, 20, shape))
    else:
        raise ValueError(dist)
    if np.issubdtype(np.dtype(dtype), np.complexfloating):
        y = rng.uniform(-1.0, 1.0, shape) if dist == "uniform" else rng.standard_normal(shape)
        return (x + 1j * y).astype(dtype)
    return x.astype(dtype)


class Problem:
    """A seeded real GEMM problem in rblas's conventions."""

    def __init__(self, layout, ta, tb, m, n, k, dtype, alpha=1.0, beta=0.0, pad=0, seed=0,
                 dist="uniform", c0_nan=False):
        rng = np.random.default_rng(seed)
        self.layout, self.ta, self.tb = layout, ta, tb
        self.m, self.n, self.k = m, n, k
        self.alpha, self.beta, self.dtype = alpha, beta, dtype
        ar, ac = stored_shape(layout, ta, m, k)
        br, bc = stored_shape(layout, tb, k, n)
        contig = lambda r, c: r if layout == 1 else c
        self.lda = max(contig(ar, ac), 1) + pad
        self.ldb = max(contig(br, bc), 1) + pad
        self.ldc = max(contig(m, n), 1) + pad
        self.a, self.A = make_buffer(rng, layout, ar, ac, self.lda, dtype, dist)
        self.b, self.B = make_buffer(rng, layout, br, bc, self.ldb, dtype, dist)
        self.c0, self.C0 = make_buffer(rng, layout, m, n, self.ldc, dtype, dist)
        if c0_nan and self.c0.size:
            oracle.stored_2d(self.c0, m, n, self.ldc, layout)[...] = np.nan
            self.C0 = np.full((m, n), np.nan, dtype)

    def opA(self):
        return self.A.T if self.ta else self.A

    def opB(self):
        return self.B.T if self.tb else self.B

    def fresh_c(self):
        return self.c0.copy()

    def result(self, c):
        return np.array(oracle.stored_2d(c, self.m, self.n, self.ldc, self.layout))

    def reference_restatement(self, threads=None):
        c = self.fresh_c()
        oracle.gemm(self.layout, int(self.ta), int(self.tb), self.m, self.n, self.k, self.alpha,
                    self.a, self.lda, self.b, self.ldb, self.beta, c, self.ldc, threads=threads)
        return c

    def dd(self, rows=None):
        return oracle.dd_gemm(self.layout, int(self.ta), int(self.tb), self.m, self.n, self.k,
                              self.alpha, self.a, self.lda, self.b, self.ldb, self.beta, self.c0,
                              self.ldc, rows=rows)

    def denom(self):
        an = np.linalg.norm(self.A.astype(np.float64)) if self.A.size else 0.0
        bn = np.linalg.norm(self.B.astype(np.float64)) if self.B.size else 0.0
        cn = np.linalg.norm(self.C0.astype(np.float64)) if (self.beta != 0 and self.C0.size) else 0.0
        return abs(self.alpha) * an * bn + abs(self.beta) * cn

    def normwise(self, c, c_ref):
        """||C - C_ref||_F / (|alpha| ||A|| ||B|| + |beta| ||C0||)."""
        d = self.result(c).astype(np.float64) - self.result(c_ref).astype(np.float64)
        den = self.denom()
        num = float(np.sqrt(np.sum(d * d)))
        return num / den if den > 0 else num

    def normwise_vs_dd(self, c, rows=None):
        hi, lo = self.dd(rows)
        r = self.result(c)
        if rows is not None:
            r = r[rows]
        diff = (r.astype(np.float64) - hi) - lo
        den = self.denom()
        if rows is not None:  # scale the denominator to the sampled rows
            an = np.linalg.norm(self.opA()[rows].astype(np.float64))
            bn = np.linalg.norm(self.B.astype(np.float64))
            cn = np.linalg.norm(self.C0.astype(np.float64)[rows]) if self.beta != 0 else 0.0
            den = abs(self.alpha) * an * bn + abs(self.beta) * cn
        num = float(np.sqrt(np.sum(diff * diff)))
        return num / den if den > 0 else num

    def tol(self):
        return 4 * max(self.k, 1) * oracle.unit_roundoff(self.dtype)
