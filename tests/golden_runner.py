"""Replays the reference's own test cases (tests/golden/ref_cases.*) against a
backend: the oracle or the GPU library's Python mirror of rblas's API.

A backend is any object exposing rblas-shaped calls:
    gemm(layout, transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
    cgemm(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
    syrk(uplo, trans, n, k, alpha, a, lda, beta, c, ldc)
    symm(side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc)
    hemm(side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc)
    trsm(side, uplo, trans, diag, m, n, alpha, a, lda, b, ldb)   (real or complex by dtype)
    check_gemm(layout, transa, transb, m, n, k, lda, a_len, ldb, b_len, ldc, c_len)
        -> (code, which, got, min_or_need)
"""
from __future__ import annotations

import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")

_DT = {"f32": np.float32, "f64": np.float64, "c32": np.complex64, "c64": np.complex128}


def load_cases():
    with open(os.path.join(GOLDEN, "ref_cases.json")) as f:
        cases = json.load(f)
    arrs = np.load(os.path.join(GOLDEN, "ref_cases.npz"))
    out = {}
    for name, meta in cases.items():
        data = {key.split("__", 1)[1]: arrs[key] for key in arrs.files if key.startswith(name + "__")}
        out[name] = (meta, data)
    return out


def _cx(v):
    return complex(v[0], v[1]) if isinstance(v, (list, tuple)) else v


def run_case(backend, meta, data, dtype_override=None):
    """Run one case; returns (ok: bool, detail: str)."""
    op = meta["op"]
    if op == "try_gemm":
        for call in meta["calls"]:
            code, which, got, need = backend.check_gemm(
                1, 0, 0, meta["m"], meta["n"], meta["k"], call["lda"], call["a_len"], call["ldb"],
                call["b_len"], call["ldc"], call["c_len"])
            w = call["want"]
            if code != w["code"]:
                return False, f"code {code} != {w['code']}"
            if code and (which != w["which"] or got != w["got"] or need != w["min_or_need"]):
                return False, f"error fields {(which, got, need)} != {w}"
        return True, "ok"
    if op == "cmul":
        return True, "host-only"
    dt = _DT[dtype_override or meta["dtype"]]
    a = np.ascontiguousarray(data["a"]).astype(dt)
    want = data["want"]
    if op == "gemm":
        b = data["b"].astype(dt)
        c = data["c0"].astype(dt).copy()
        backend.gemm(meta["layout"], meta["transa"], meta["transb"], meta["m"], meta["n"],
                     meta["k"], meta["alpha"], a, meta["lda"], b, meta["ldb"], meta["beta"], c,
                     meta["ldc"])
        got = c
    elif op == "cgemm":
        b = data["b"].astype(dt)
        c = data["c0"].astype(dt).copy()
        backend.cgemm(meta["transa"], meta["transb"], meta["m"], meta["n"], meta["k"],
                      _cx(meta["alpha"]), a, meta["lda"], b, meta["ldb"], _cx(meta["beta"]), c,
                      meta["ldc"])
        got = c
    elif op == "syrk":
        c = data["c0"].astype(dt).copy()
        backend.syrk(meta["uplo"], meta["trans"], meta["n"], meta["k"], meta["alpha"], a,
                     meta["lda"], meta["beta"], c, meta["ldc"])
        got = c
    elif op in ("symm", "hemm"):
        b = data["b"].astype(dt)
        c = data["c0"].astype(dt).copy()
        fn = backend.symm if op == "symm" else backend.hemm
        fn(meta["side"], meta["uplo"], meta["m"], meta["n"], _cx(meta["alpha"]), a, meta["lda"], b,
           meta["ldb"], _cx(meta["beta"]), c, meta["ldc"])
        got = c
    elif op in ("trsm", "ctrsm"):
        b = data["b"].astype(dt).copy()
        backend.trsm(meta["side"], meta["uplo"], meta["trans"], meta["diag"], meta["m"], meta["n"],
                     _cx(meta["alpha"]), a, meta["lda"], b, meta["ldb"])
        got = b
    else:
        raise ValueError(op)
    return _compare(meta, data, got, want, a)


def _compare(meta, data, got, want, a):
    chk, tol = meta["check"], meta["tol"]
    got = np.asarray(got)
    if chk == "exact":
        ok = np.array_equal(got.astype(want.dtype), want)
        return ok, f"got {got} want {want}"
    if chk == "abs":
        err = np.max(np.abs(got.astype(np.complex128 if np.iscomplexobj(got) else np.float64) - want))
        return err < tol, f"max abs err {err:.3e} tol {tol}"
    if chk == "cabs_parts":
        g = got.astype(np.complex128)
        err = max(np.max(np.abs(g.real - want.real)), np.max(np.abs(g.imag - want.imag)))
        return err < tol, f"max part err {err:.3e} tol {tol}"
    if chk == "cabs":
        err = np.max(np.abs(got.astype(np.complex128) - want))
        return err < tol, f"max |err| {err:.3e} tol {tol}"
    if chk == "spot00":
        err = abs(float(got[0]) - float(want[0]))
        exact_all = np.array_equal(got, want.astype(got.dtype))
        return err < tol and exact_all, f"c[0] err {err:.3e}; all-entries exact={exact_all}"
    if chk == "maxrel":
        w = want.astype(np.float32)
        denom = np.maximum(np.abs(w), np.float32(meta["denom_floor"]))
        rel = float(np.max(np.abs(got - w) / denom))
        return rel < tol, f"max rel {rel:.3e} tol {tol}"
    if chk == "tri_abs":
        n = meta["n"]
        G = got.reshape(n, n).T
        W = want.reshape(n, n).T
        mask = np.tril(np.ones((n, n), bool)) if meta["uplo"] == 1 else np.triu(np.ones((n, n), bool))
        err = float(np.max(np.abs(G[mask] - W[mask])))
        return err < tol, f"max tri err {err:.3e} tol {tol}"
    if chk == "roundtrip_right":
        m, n = meta["m"], meta["n"]
        X = got.reshape(n, m).T.astype(np.float64)
        U = data["a"].reshape(n, n).T
        B0 = want.reshape(n, m).T
        R = np.zeros((m, n))
        for i in range(m):
            for j in range(n):
                s = 0.0
                for kk in range(n):
                    s += X[i, kk] * U[kk, j]
                R[i, j] = s
        err = float(np.max(np.abs(R - B0)))
        return err < tol, f"roundtrip err {err:.3e}"
    if chk == "roundtrip_left_lower":
        m = meta["m"]
        L = data["a"].reshape(m, m).T
        x = got.astype(np.complex128)
        errs = []
        for i in range(m):
            s = 0j
            for j in range(i + 1):
                s += L[i, j] * x[j]
            errs.append(abs(s - want[i]))
        err = max(errs)
        return err < tol, f"roundtrip err {err:.3e}"
    raise ValueError(chk)
