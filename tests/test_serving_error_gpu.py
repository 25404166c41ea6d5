"""Per-request error of the serving configuration against the FP64 oracle.

A 512-request slice of the serving stream -- m, n, k log-uniform in
[32, 4096], dtype 50/50 f32/f64, layout and transposes uniform, alpha and
beta uniform in [-2, 2], standard-normal operands resident in HBM -- runs
through the serving loop (rb_server_*) in three modes: grouped plain, grouped
with the precision forms for large requests (BF16X6 for f32 requests of at
least 2e8 flop, Ozaki for f64 requests of at least 1e9 flop, the rest grouped
plain), and one plain launch per request. Every request of every mode is
compared with the double-double oracle (oracle.dd_core) on a seeded sample of
16 rows of C (all rows when C has fewer), each call of rblas's gemm
(level3::gemm, src/level3.rs:32-62) that the request stands for.

Tolerances, per request (u of the request's dtype):
  * plain (grouped and per-request): normwise error <= 4*k*u.
  * a request the forms mode runs in a precision form: <= 4*k*u and
    <= 2 x the same request's per-request plain error + u/16 (the sample's
    rounding noise floor). Requests it keeps plain: as plain.
The distribution (median / max error and form-vs-plain ratio per mode) is
written to the file named by RB_SERVING_ERROR_REPORT when that is set.
"""
from __future__ import annotations

import json
import os

import numpy as np
import pytest

import oracle
from rblas_b200.serving import Problem, Server

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

N_REQ = 512
SAMPLE_ROWS = 16
FORMS = {"f32_form": 3, "f64_form": 2, "f32_min_flop": 2e8, "f64_min_flop": 1e9}
POOL = 4096 * 4096 + (1 << 22)


def _stream(seed=5):
    rng = np.random.default_rng(seed)
    mnk = np.exp(rng.uniform(np.log(32), np.log(4096), (N_REQ, 3))).astype(np.int64)
    return dict(mnk=mnk, dtype=rng.integers(0, 2, N_REQ), layout=rng.integers(0, 2, N_REQ),
                ta=rng.integers(0, 3, N_REQ), tb=rng.integers(0, 3, N_REQ),
                alpha=rng.uniform(-2, 2, N_REQ), beta=rng.uniform(-2, 2, N_REQ),
                offs=rng.integers(0, 1 << 20, (N_REQ, 3)), rows=rng.integers(0, 1 << 30, N_REQ))


def _stored(pool, off, rows, cols, ld, layout):
    """The stored rows x cols matrix at element offset `off` of a pool."""
    if layout == 1:
        return torch.as_strided(pool, (rows, cols), (1, ld), off)
    return torch.as_strided(pool, (rows, cols), (ld, 1), off)


def _requests(pools, tr):
    out = []
    for i in range(N_REQ):
        m, n, k = (int(x) for x in tr["mnk"][i])
        dt = int(tr["dtype"][i])
        vec = 4 if dt == 0 else 2
        layout, ta, tb = int(tr["layout"][i]), int(tr["ta"][i]), int(tr["tb"][i])
        ar, ac = (k, m) if ta else (m, k)
        br, bc = (n, k) if tb else (k, n)
        pad = lambda x: (x + vec - 1) // vec * vec  # noqa: E731
        lda = pad(ar) if layout == 1 else pad(ac)
        ldb = pad(br) if layout == 1 else pad(bc)
        ldc = pad(m) if layout == 1 else pad(n)
        es = 4 if dt == 0 else 8
        offs = [int(o) // 16 * 16 for o in tr["offs"][i]]
        base = pools[dt].data_ptr()
        p = Problem(np.float32 if dt == 0 else np.float64, layout, ta, tb, m, n, k, float(tr["alpha"][i]),
                    base + offs[0] * es, lda, base + offs[1] * es, ldb, float(tr["beta"][i]), base + offs[2] * es,
                    ldc)
        out.append((p, offs, (ar, ac), (br, bc)))
    return out


def _reference(pools, req, rows):
    """(hi + lo of the double-double result on `rows`, row-scaled denominator)."""
    p, offs, (ar, ac), (br, bc) = req
    pool = pools[0 if p.dtype == np.float32 else 1]
    A = _stored(pool, offs[0], ar, ac, p.lda, p.layout)
    B = _stored(pool, offs[1], br, bc, p.ldb, p.layout)
    C0 = _stored(pool, offs[2], p.m, p.n, p.ldc, p.layout)
    opA = (A.t() if p.transa else A)[rows].double().cpu().numpy()
    opB = (B.t() if p.transb else B).double().cpu().numpy()
    c0 = C0[rows].double().cpu().numpy()
    hi, lo = oracle.dd_core(opA, opB, p.alpha, p.beta, c0 if p.beta != 0 else None)
    den = abs(p.alpha) * np.linalg.norm(opA) * np.linalg.norm(opB) + abs(p.beta) * np.linalg.norm(c0)
    return hi, lo, den


def _result_rows(p, d, ldd, rows):
    rs, cs = (p.m, p.n) if p.layout == 1 else (p.n, p.m)

    class _View:
        __cuda_array_interface__ = {"shape": (ldd * cs,), "typestr": np.dtype(p.dtype).str, "data": (d, False),
                                    "version": 3}

    flat = torch.as_tensor(_View(), device="cuda")
    D = torch.as_strided(flat, (p.m, p.n), (1, ldd) if p.layout == 1 else (ldd, 1))
    return D[rows].double().cpu().numpy()


def _serve(reqs, rows, grouped, forms):
    """Submit every request, then read each result's sampled rows."""
    got = []
    with Server(budget_bytes=24 << 30, max_batch=256, grouped=grouped) as srv:
        if forms:
            srv.set_forms(**FORMS)
        ids = [srv.submit(r[0]) for r in reqs]
        for rid, r, rw in zip(ids, reqs, rows):
            st, d, ldd, _ = srv.wait(rid)
            assert st == 0, (st, r[0].m, r[0].n, r[0].k)
            got.append(_result_rows(r[0], d, ldd, rw))
            srv.release(rid)
    return got


def _in_form(p):
    flop = 2.0 * p.m * p.n * p.k
    if p.dtype == np.float32:
        return flop >= FORMS["f32_min_flop"]
    return flop >= FORMS["f64_min_flop"]


def test_serving_stream_per_request_error_vs_fp64_oracle():
    tr = _stream()
    g = torch.Generator(device="cuda")
    g.manual_seed(5)
    pools = {0: torch.randn(POOL, dtype=torch.float32, device="cuda", generator=g),
             1: torch.randn(POOL, dtype=torch.float64, device="cuda", generator=g)}
    reqs = _requests(pools, tr)
    rows = []
    for i, (p, *_rest) in enumerate(reqs):
        r = np.random.default_rng(int(tr["rows"][i]))
        rows.append(np.sort(r.choice(p.m, min(SAMPLE_ROWS, p.m), replace=False)))
    refs = [_reference(pools, req, rw) for req, rw in zip(reqs, rows)]
    modes = {"grouped": (True, False), "per_request": (False, False), "grouped_forms": (True, True)}
    errs = {}
    for mode, (grouped, forms) in modes.items():
        got = _serve(reqs, rows, grouped, forms)
        e = []
        for (hi, lo, den), gv in zip(refs, got):
            diff = (gv - hi) - lo
            num = float(np.sqrt(np.sum(diff * diff)))
            e.append(num / den if den > 0 else num)
        errs[mode] = np.array(e)
    u = np.array([2.0 ** -24 if r[0].dtype == np.float32 else 2.0 ** -53 for r in reqs])
    k = np.array([max(r[0].k, 1) for r in reqs], dtype=np.float64)
    in_form = np.array([_in_form(r[0]) for r in reqs])
    f32 = np.array([r[0].dtype == np.float32 for r in reqs])
    report = {"requests": N_REQ, "sample_rows": SAMPLE_ROWS, "forms": FORMS,
              "in_form": {"f32": int(np.sum(in_form & f32)), "f64": int(np.sum(in_form & ~f32))}}
    bound = 4 * k * u
    for mode, e in errs.items():
        sel = {"f32": f32, "f64": ~f32}
        report[mode] = {dt: {"median": float(np.median(e[s])), "max": float(np.max(e[s])),
                             "max_over_bound": float(np.max(e[s] / bound[s]))} for dt, s in sel.items()}
    ratio = errs["grouped_forms"] / np.maximum(errs["per_request"], 1e-300)
    for dt, s in (("f32", f32), ("f64", ~f32)):
        sf = in_form & s
        if np.any(sf):
            report["grouped_forms"][dt]["form_vs_plain_ratio"] = {
                "median": float(np.median(ratio[sf])), "max": float(np.max(ratio[sf]))}
    path = os.environ.get("RB_SERVING_ERROR_REPORT")
    if path:
        with open(path, "w") as f:
            json.dump(report, f, indent=1)
    print(json.dumps(report, indent=1))
    for mode, e in errs.items():
        bad = np.nonzero(e > bound)[0]
        assert bad.size == 0, (mode, [(reqs[i][0].m, reqs[i][0].n, reqs[i][0].k, e[i], bound[i]) for i in bad[:5]])
    lim = 2 * errs["per_request"] + u / 16
    bad = np.nonzero(in_form & (errs["grouped_forms"] > lim))[0]
    assert bad.size == 0, [(reqs[i][0].m, reqs[i][0].n, reqs[i][0].k, str(reqs[i][0].dtype),
                            errs["grouped_forms"][i], errs["per_request"][i]) for i in bad[:8]]
