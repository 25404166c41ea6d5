"""Generate tests/golden/ref_cases.npz + ref_cases.json.

Each case restates one test of the reference (blasrodri/rblas) exactly as its
source builds it: the same fills (sin/cos closed forms, the LCG of
tests/correctness.rs:21-26 and tests/parallel.rs:9-14), the same call, and the
expected values the reference test computes with its own naive formulas
(sequential, unfused `acc += a*b` in the test's precision; numpy ops round once
per operation like the Rust expressions). The tolerance and comparison of the
reference assertion travel with the case. The reference itself cannot be built
here (Rust toolchain absent), so these are the vectors that pin the oracle and
the GPU library to the reference's tested behaviour.

Run:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
A6364 = np.uint64(6364136223846793005)
C1442 = np.uint64(1442695040888963407)


def lcg(seed: int, n: int, mode: int) -> np.ndarray:
    """tests/correctness.rs:21-26 (mode 0) / tests/parallel.rs:9-14 (mode 1)."""
    out = np.empty(n, dtype=np.float32)
    s = np.uint64(seed)
    with np.errstate(over="ignore"):
        for i in range(n):
            s = s * A6364 + C1442
            if mode == 0:
                v = np.float32(int(s) >> 33)
                out[i] = np.float32(v / np.float32(2.0 ** 31)) - np.float32(1.0)
            else:
                v = np.float32(int(s) >> 40)
                out[i] = np.float32(v / np.float32(2.0 ** 24)) - np.float32(0.5)
    return out


def naive_colmajor(m, n, k, a, b, dtype, at=None, bt=None):
    """Sequential unfused acc += a*b, as the reference tests' naive loops."""
    A = at if at is not None else a.reshape(k, m).T  # [i, p]
    B = bt if bt is not None else b.reshape(n, k).T  # [p, j]
    acc = np.zeros((m, n), dtype=dtype)
    for p in range(k):
        acc = (acc + (A[:, p:p + 1] * B[p:p + 1, :]).astype(dtype)).astype(dtype)
    return acc.T.reshape(-1).copy()  # col-major flat


def cnaive(m, n, k, A, B):
    """Complex naive loop acc = acc + a*b with rblas Complex arithmetic
    (src/complex.rs:101-111: re = fma(a.re,b.re,-(a.im*b.im)), im = fma(a.re,b.im,a.im*b.re)).
    fma is evaluated exactly then rounded (via extended products in float64
    with two-product correction is unnecessary here: reference checks at 1e-9)."""
    acc = np.zeros((m, n), dtype=np.complex128)
    for p in range(k):
        acc = acc + A[:, p:p + 1] * B[p:p + 1, :]
    return acc


cases = {}
arrays = {}


def add(name, meta, **arrs):
    cases[name] = meta
    for key, v in arrs.items():
        arrays[f"{name}__{key}"] = np.asarray(v)


# --- src/kernel/gemm.rs:690-701 gemm_matches_reference ---------------------
m, n, k = 17, 13, 19
a = np.sin(np.arange(m * k) * 0.5)
b = np.cos(np.arange(k * n) * 0.3)
add("gemm_matches_reference",
    dict(ref="src/kernel/gemm.rs:690-701", op="gemm", dtype="f64", layout=1, transa=0, transb=0,
         m=m, n=n, k=k, alpha=1.0, beta=0.0, lda=m, ldb=k, ldc=m, check="abs", tol=1e-9),
    a=a, b=b, c0=np.zeros(m * n), want=naive_colmajor(m, n, k, a, b, np.float64))

# --- src/kernel/gemm.rs:704-717 gemm_alpha_beta -----------------------------
m = n = k = 8
a = np.arange(m * k, dtype=np.float32)
b = (np.arange(k * n) % 5).astype(np.float32)
want = (2.0 * naive_colmajor(m, n, k, a, b, np.float64) + 3.0).astype(np.float32)
add("gemm_alpha_beta",
    dict(ref="src/kernel/gemm.rs:704-717", op="gemm", dtype="f32", layout=1, transa=0, transb=0,
         m=m, n=n, k=k, alpha=2.0, beta=3.0, lda=m, ldb=k, ldc=m, check="spot00", tol=1e-3),
    a=a, b=b, c0=np.ones(m * n, dtype=np.float32), want=want)

# --- src/level3.rs:567-640 try_gemm_ok_and_errors ----------------------------
add("try_gemm_errors",
    dict(ref="src/level3.rs:567-640", op="try_gemm", dtype="f64", m=4, n=3, k=5,
         calls=[
             dict(lda=4, a_len=20, ldb=5, b_len=15, ldc=4, c_len=12, want=dict(code=0)),
             dict(lda=3, a_len=20, ldb=5, b_len=15, ldc=4, c_len=12,
                  want=dict(code=1, which="a", got=3, min_or_need=4)),
             dict(lda=4, a_len=20, ldb=5, b_len=15, ldc=4, c_len=11,
                  want=dict(code=2, which="c", got=11, min_or_need=12)),
         ]))

# --- src/level3.rs:643-667 gemm_nn_colmajor ---------------------------------
m, n, k = 6, 5, 7
a = np.arange(m * k, dtype=np.float64)
b = np.arange(k * n, dtype=np.float64) * 2
add("gemm_nn_colmajor",
    dict(ref="src/level3.rs:643-667", op="gemm", dtype="f64", layout=1, transa=0, transb=0,
         m=m, n=n, k=k, alpha=1.0, beta=0.0, lda=m, ldb=k, ldc=m, check="abs", tol=1e-9),
    a=a, b=b, c0=np.zeros(m * n), want=naive_colmajor(m, n, k, a, b, np.float64))

# --- src/level3.rs:669-694 gemm_tn_colmajor ---------------------------------
m, n, k = 4, 5, 6
a = np.sqrt(np.arange(k * m, dtype=np.float64))
b = np.arange(k * n, dtype=np.float64) * 0.1
At = a.reshape(m, k)  # stored k x m col-major: a[p + i*k] -> At[i, p]
add("gemm_tn_colmajor",
    dict(ref="src/level3.rs:669-694", op="gemm", dtype="f64", layout=1, transa=1, transb=0,
         m=m, n=n, k=k, alpha=1.0, beta=0.0, lda=k, ldb=k, ldc=m, check="abs", tol=1e-9),
    a=a, b=b, c0=np.zeros(m * n), want=naive_colmajor(m, n, k, None, b, np.float64, at=At))

# --- src/level3.rs:696-731 gemm_rowmajor_nn ---------------------------------
m, n, k = 5, 4, 3
a = np.arange(m * k, dtype=np.float64)
b = np.arange(k * n, dtype=np.float64) + 1
A = a.reshape(m, k)
B = b.reshape(k, n)
acc = np.zeros((m, n))
for p in range(k):
    acc = acc + A[:, p:p + 1] * B[p:p + 1, :]
add("gemm_rowmajor_nn",
    dict(ref="src/level3.rs:696-731", op="gemm", dtype="f64", layout=0, transa=0, transb=0,
         m=m, n=n, k=k, alpha=1.0, beta=0.0, lda=k, ldb=n, ldc=n, check="abs", tol=1e-9),
    a=a, b=b, c0=np.zeros(m * n), want=acc.reshape(-1))

# --- src/level3.rs:733-759 syrk_lower_notrans -------------------------------
n, k = 3, 2
a = np.array([1.0, 2, 3, 4, 5, 6])
Aem = a.reshape(k, n).T
full = np.zeros((n, n))
for p in range(k):
    full = full + Aem[:, p:p + 1] * Aem[:, p:p + 1].T
add("syrk_lower_notrans",
    dict(ref="src/level3.rs:733-759", op="syrk", dtype="f64", uplo=1, trans=0, n=n, k=k,
         alpha=1.0, beta=0.0, lda=n, ldc=n, check="tri_abs", tol=1e-12),
    a=a, c0=np.zeros(n * n), want=full.T.reshape(-1))

# --- src/level3.rs:761-792 symm_left_upper (exact) ---------------------------
add("symm_left_upper",
    dict(ref="src/level3.rs:761-792", op="symm", dtype="f64", side=0, uplo=0, m=2, n=2,
         alpha=1.0, beta=0.0, lda=2, ldb=2, ldc=2, check="exact", tol=0.0),
    a=np.array([2.0, 0.0, 1.0, 3.0]), b=np.array([1.0, 2.0, 3.0, 4.0]), c0=np.zeros(4),
    want=np.array([4.0, 7.0, 10.0, 15.0]))

# --- src/level3.rs:794-825 syrk_trans_upper_larger ---------------------------
n, k = 9, 11
a = np.sin(np.arange(k * n) * 0.31)
c0 = np.arange(n * n) * 0.1
Ast = a.reshape(n, k).T  # A[p, i] = a[p + i*k]
want = c0.copy()
for j in range(n):
    for i in range(j + 1):
        acc = 0.0
        for p in range(k):
            acc += Ast[p, i] * Ast[p, j]
        want[i + j * n] = 2.0 * acc + 3.0 * c0[i + j * n]
add("syrk_trans_upper_larger",
    dict(ref="src/level3.rs:794-825", op="syrk", dtype="f64", uplo=0, trans=1, n=n, k=k,
         alpha=2.0, beta=3.0, lda=k, ldc=n, check="tri_abs", tol=1e-9),
    a=a, c0=c0, want=want)

# --- src/level3.rs:827-866 symm_right_lower_larger ---------------------------
m, n = 7, 6
al = np.cos(np.arange(n * n) * 0.17)
b = np.arange(m * n) * 0.05
want = np.zeros(m * n)
sym = lambda i, j: al[i + j * n] if i >= j else al[j + i * n]
for j in range(n):
    for i in range(m):
        acc = 0.0
        for p in range(n):
            acc += b[i + p * m] * sym(p, j)
        want[i + j * m] = acc
add("symm_right_lower_larger",
    dict(ref="src/level3.rs:827-866", op="symm", dtype="f64", side=1, uplo=1, m=m, n=n,
         alpha=1.0, beta=0.0, lda=n, ldb=m, ldc=m, check="abs", tol=1e-9),
    a=al, b=b, c0=np.zeros(m * n), want=want)

# --- src/level3.rs:868-903 trsm_left_lower_notrans ---------------------------
L = np.array([2.0, 1, 1, 0, 3, 2, 0, 0, 4])
xtrue = np.array([1.0, 2.0, 3.0])
bb = np.zeros(3)
for i in range(3):
    s = 0.0
    for j in range(i + 1):
        s += L[i + j * 3] * xtrue[j]
    bb[i] = s
add("trsm_left_lower_notrans",
    dict(ref="src/level3.rs:868-903", op="trsm", dtype="f64", side=0, uplo=1, trans=0, diag=0,
         m=3, n=1, alpha=1.0, lda=3, ldb=3, check="abs", tol=1e-12),
    a=L, b=bb, want=xtrue)

# --- src/level3.rs:905-934 trsm_right_upper_roundtrip ------------------------
add("trsm_right_upper_roundtrip",
    dict(ref="src/level3.rs:905-934", op="trsm", dtype="f64", side=1, uplo=0, trans=0, diag=0,
         m=2, n=3, alpha=1.0, lda=3, ldb=2, check="roundtrip_right", tol=1e-10),
    a=np.array([2.0, 0, 0, 1, 3, 0, 4, 5, 6]), b=np.array([1.0, 4, 2, 5, 3, 6]),
    want=np.array([1.0, 4, 2, 5, 3, 6]))

# --- src/complex3.rs:372-401 gemm_matches_naive ------------------------------
m, n, k = 5, 4, 6
ia = np.arange(m * k)
ib = np.arange(k * n)
ca = np.sin(ia * 0.3) + 1j * np.cos(ia * 0.7)
cb = np.cos(ib * 0.2) + 1j * np.sin(ib * 0.5)
want = cnaive(m, n, k, ca.reshape(k, m).T, cb.reshape(n, k).T).T.reshape(-1)
add("cgemm_matches_naive",
    dict(ref="src/complex3.rs:372-401", op="cgemm", dtype="c64", transa=0, transb=0, m=m, n=n,
         k=k, alpha=[1.0, 0.0], beta=[0.0, 0.0], lda=m, ldb=k, ldc=m, check="cabs_parts",
         tol=1e-9),
    a=ca, b=cb, c0=np.zeros(m * n, dtype=np.complex128), want=want)

# --- src/complex3.rs:403-437 gemm_conjtrans_a --------------------------------
m, n, k = 3, 2, 4
ia = np.arange(k * m)
ca = ia + 1j * (ia * 0.5)
cb = np.ones(k * n) + 1j * np.arange(k * n)
Aop = np.conj(ca.reshape(m, k))  # op(A)[i,p] = conj(a[p + i*k])
want = cnaive(m, n, k, Aop, cb.reshape(n, k).T).T.reshape(-1)
add("cgemm_conjtrans_a",
    dict(ref="src/complex3.rs:403-437", op="cgemm", dtype="c64", transa=2, transb=0, m=m, n=n,
         k=k, alpha=[1.0, 0.0], beta=[0.0, 0.0], lda=k, ldb=k, ldc=m, check="cabs", tol=1e-9),
    a=ca, b=cb, c0=np.zeros(m * n, dtype=np.complex128), want=want)

# --- src/complex3.rs:439-477 trsm_left_lower_roundtrip -----------------------
Lc = np.array([2 + 1j, 1 + 0j, 0.5 - 1j, 0, 3 - 1j, 1 + 1j, 0, 0, 4 + 0.5j])
b0 = np.array([1 + 1j, 2 + 0j, 0 + 3j])
add("ctrsm_left_lower_roundtrip",
    dict(ref="src/complex3.rs:439-477", op="ctrsm", dtype="c64", side=0, uplo=1, trans=0, diag=0,
         m=3, n=1, alpha=[1.0, 0.0], lda=3, ldb=3, check="roundtrip_left_lower", tol=1e-9),
    a=Lc, b=b0, want=b0)

# --- src/complex3.rs:479-509 hemm_left_upper (exact) -------------------------
add("hemm_left_upper",
    dict(ref="src/complex3.rs:479-509", op="hemm", dtype="c64", side=0, uplo=0, m=2, n=1,
         alpha=[1.0, 0.0], beta=[0.0, 0.0], lda=2, ldb=2, ldc=2, check="cabs", tol=1e-12),
    a=np.array([2 + 0j, 9 + 9j, 1 + 1j, 3 + 0j]), b=np.array([1 + 0j, 0 + 1j]),
    c0=np.zeros(2, dtype=np.complex128), want=np.array([1 + 1j, 1 + 2j]))

# --- src/complex3.rs:511-558 hemm_left_lower_larger --------------------------
q, n = 5, 3
ia = np.arange(q * q)
ib = np.arange(q * n)
ca = np.sin(ia * 0.3) + 1j * np.cos(ia * 0.4)
cb = ib * 0.1 + 1j * (ib * 0.05)


def her(i, j):
    if i > j:
        return ca[i + j * q]
    if i < j:
        return np.conj(ca[j + i * q])
    return complex(ca[i + j * q].real, 0.0)


alpha = 1.5 - 0.5j
want = np.zeros(q * n, dtype=np.complex128)
for j in range(n):
    for i in range(q):
        acc = 0j
        for p in range(q):
            acc = acc + her(i, p) * cb[p + j * q]
        want[i + j * q] = alpha * acc
add("hemm_left_lower_larger",
    dict(ref="src/complex3.rs:511-558", op="hemm", dtype="c64", side=0, uplo=1, m=q, n=n,
         alpha=[1.5, -0.5], beta=[0.0, 0.0], lda=q, ldb=q, ldc=q, check="cabs", tol=1e-9),
    a=ca, b=cb, c0=np.zeros(q * n, dtype=np.complex128), want=want)

# --- src/complex.rs:122-130 mul_and_conj (exact) ------------------------------
add("complex_mul",
    dict(ref="src/complex.rs:122-130", op="cmul", check="exact", tol=0.0),
    a=np.array([1 + 2j]), b=np.array([3 - 1j]), want=np.array([5 + 5j]))

# --- tests/correctness.rs:28-58 large_random_sgemm_matches_naive --------------
m, n, k = 200, 180, 150
vals = lcg(0x12345678, m * k + k * n, 0)
a, b = vals[:m * k], vals[m * k:]
add("correctness_large_random_sgemm",
    dict(ref="tests/correctness.rs:28-58", op="gemm", dtype="f32", layout=1, transa=0, transb=0,
         m=m, n=n, k=k, alpha=1.0, beta=0.0, lda=m, ldb=k, ldc=m, check="maxrel", tol=1e-3,
         denom_floor=1e-4),
    a=a, b=b, c0=np.zeros(m * n, dtype=np.float32), want=naive_colmajor(m, n, k, a, b, np.float32))

# --- tests/parallel.rs:16-63 parallel_matches_serial ----------------------------
m, n, k = 64, 5000, 48
vals = lcg(0xC0FFEE, m * k + k * n, 1)
a, b = vals[:m * k], vals[m * k:]
add("parallel_matches_serial",
    dict(ref="tests/parallel.rs:16-63", op="gemm", dtype="f32", layout=1, transa=0, transb=0,
         m=m, n=n, k=k, alpha=1.0, beta=0.0, lda=m, ldb=k, ldc=m, check="maxrel", tol=1e-2,
         denom_floor=1e-3),
    a=a, b=b, c0=np.zeros(m * n, dtype=np.float32), want=naive_colmajor(m, n, k, a, b, np.float32))

if __name__ == "__main__":
    np.savez_compressed(os.path.join(HERE, "ref_cases.npz"), **arrays)
    with open(os.path.join(HERE, "ref_cases.json"), "w") as f:
        json.dump(cases, f, indent=1, sort_keys=True)
    print(f"wrote {len(cases)} cases, {len(arrays)} arrays")
