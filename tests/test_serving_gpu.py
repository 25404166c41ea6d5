"""GPU tests of the batching and serving forms: the grouped persistent kernel
(rb_gemm_grouped_dev) and the serving loop (rb_server_*), called through the
C ABI on device-resident operands and checked against the oracle and against
the single-problem entry point.

Tolerance: every result within 4*k*u (u of its dtype) normwise of the
restatement of rblas's gemm; the grouped kernel runs the same tile code as
the single-problem kernel, so those two agree exactly, and a request's
result is exactly the same alone and in a mix.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from rblas_b200 import level3
from rblas_b200.serving import GroupedPlan, Problem, Server, grouped_gemm, grouped_splits
from rblas_b200.types import Layout

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _tdt(dt):
    return torch.float32 if np.dtype(dt) == np.float32 else torch.float64


def make_problem(rng, dt, layout, ta, tb, m, n, k, alpha, beta):
    ar, ac = (k, m) if ta else (m, k)
    br, bc = (n, k) if tb else (k, n)
    contig = (lambda r, c: r) if layout == Layout.ColMajor else (lambda r, c: c)
    lda, ldb, ldc = max(contig(ar, ac), 1), max(contig(br, bc), 1), max(contig(m, n), 1)
    A = torch.tensor(rng.standard_normal(max(ar * ac, 1)), dtype=_tdt(dt), device="cuda")
    B = torch.tensor(rng.standard_normal(max(br * bc, 1)), dtype=_tdt(dt), device="cuda")
    Cc = torch.tensor(rng.standard_normal(max(m * n, 1)), dtype=_tdt(dt), device="cuda")
    p = Problem(dt, layout, ta, tb, m, n, k, alpha, A.data_ptr(), lda, B.data_ptr(), ldb, beta,
                Cc.data_ptr(), ldc)
    return p, (A, B, Cc)


def restatement(p, A, B, C0):
    c = C0.cpu().numpy().copy()
    oracle.gemm(int(p.layout), p.transa, p.transb, p.m, p.n, p.k, p.alpha, A.cpu().numpy(), p.lda,
                B.cpu().numpy(), p.ldb, p.beta, c, p.ldc)
    return c


def normwise(p, got, ref, A, B, C0):
    d = got.astype(np.float64) - ref.astype(np.float64)
    # beta == 0: C0 is never read (it may hold NaN), so it adds nothing
    den = abs(p.alpha) * float(A.double().norm()) * float(B.double().norm()) + \
        (abs(p.beta) * float(C0.double().norm()) if p.beta != 0.0 else 0.0)
    return float(np.sqrt(np.sum(d * d))) / den if den else float(np.sqrt(np.sum(d * d)))


def random_mix(rng, count, max_dim=700):
    out = []
    for i in range(count):
        dt = [np.float32, np.float64][rng.integers(2)]
        layout = [Layout.RowMajor, Layout.ColMajor][rng.integers(2)]
        ta, tb = int(rng.integers(3)), int(rng.integers(3))
        m, n, k = (int(np.exp(rng.uniform(0, np.log(max_dim)))) for _ in range(3))
        alpha, beta = float(rng.uniform(-2, 2)), float(rng.uniform(-2, 2))
        out.append(make_problem(rng, dt, layout, ta, tb, m, n, k, alpha, beta))
    return out


def test_grouped_matches_restatement_and_single_calls():
    rng = np.random.default_rng(60)
    probs = random_mix(rng, 48)
    # split-K cases: few C tiles, long K (f32 and f64, both transposes)
    probs.append(make_problem(rng, np.float32, Layout.ColMajor, 0, 0, 100, 90, 3000, 1.25, 0.5))
    probs.append(make_problem(rng, np.float64, Layout.RowMajor, 1, 2, 130, 70, 2500, -0.75, 1.0))
    probs.append(make_problem(rng, np.float64, Layout.ColMajor, 2, 1, 257, 129, 1111, 0.5, 0.0))
    # edge cases: k == 0, alpha == 0, a 1 x 1 x 1 problem, beta == 0 with NaN C
    probs.append(make_problem(rng, np.float64, Layout.ColMajor, 0, 0, 33, 17, 0, 1.5, -0.5))
    probs.append(make_problem(rng, np.float32, Layout.RowMajor, 1, 0, 40, 21, 13, 0.0, 2.0))
    probs.append(make_problem(rng, np.float64, Layout.ColMajor, 0, 1, 1, 1, 1, 1.0, 0.0))
    p_nan, t_nan = make_problem(rng, np.float32, Layout.ColMajor, 0, 0, 50, 60, 70, 1.0, 0.0)
    t_nan[2].fill_(float("nan"))
    probs.append((p_nan, t_nan))
    c0s = [t[2].clone() for _, t in probs]
    singles = []
    for (p, (A, B, Cc)), c0 in zip(probs, c0s):
        c = c0.clone()
        level3.gemm_dev(p.layout, p.transa, p.transb, p.m, p.n, p.k, p.alpha, p.a, p.lda, p.b, p.ldb,
                        p.beta, c.data_ptr(), p.ldc, p.dtype)
        singles.append(c)
    grouped_gemm([p for p, _ in probs])
    torch.cuda.synchronize()
    for i, ((p, (A, B, Cc)), c0, single) in enumerate(zip(probs, c0s, singles)):
        got = Cc.cpu().numpy()
        if grouped_splits(p) == 1:
            # the same tile code with the same K order as the single-problem kernel
            assert np.array_equal(got, single.cpu().numpy(), equal_nan=True), f"problem {i} differs from single call"
        if p.beta == 0.0:
            assert not np.any(np.isnan(got))
        ref = restatement(p, A, B, c0)
        tol = 4 * max(p.k, 1) * (2.0 ** -24 if p.dtype == np.float32 else 2.0 ** -53)
        assert normwise(p, got, ref, A, B, c0) <= tol, f"problem {i}"


def test_grouped_split_results_independent_of_the_mix():
    """A split problem gives bit-identical results alone and in a launch
    with many others (the split factor is shape-only, the K partials are
    summed in a fixed order)."""
    rng = np.random.default_rng(64)
    target, (A, B, C0) = make_problem(rng, np.float32, Layout.ColMajor, 0, 1, 150, 200, 4000, 1.5, -1.0)
    assert grouped_splits(target) > 1
    c0 = C0.clone()
    grouped_gemm([target])
    torch.cuda.synchronize()
    alone = C0.clone()
    C0.copy_(c0)
    mix = random_mix(rng, 40)
    grouped_gemm([p for p, _ in mix[:20]] + [target] + [p for p, _ in mix[20:]])
    torch.cuda.synchronize()
    assert torch.equal(alone, C0)
    ref = restatement(target, A, B, c0)
    assert normwise(target, alone.cpu().numpy(), ref, A, B, c0) <= 4 * 4000 * 2.0 ** -24


def test_grouped_plan_graph_replay_matches_one_shot_launch():
    """A plan (CUDA graph) replayed twice, with new operand contents before
    the second replay, gives bit-identical results to one-shot grouped
    launches on the same data (same table order, same split-K)."""
    rng = np.random.default_rng(65)
    probs = random_mix(rng, 24)
    probs.append(make_problem(rng, np.float64, Layout.ColMajor, 0, 0, 96, 80, 3000, 1.0, 1.0))  # split-K
    # an operand TMA cannot address directly (odd leading dimension): repacked in the graph
    m, n, k = 70, 50, 33
    A = torch.tensor(rng.standard_normal(71 * k), dtype=torch.float32, device="cuda")
    B = torch.tensor(rng.standard_normal(k * n), dtype=torch.float32, device="cuda")
    Cc = torch.tensor(rng.standard_normal(m * n), dtype=torch.float32, device="cuda")
    probs.append((Problem(np.float32, Layout.ColMajor, 0, 0, m, n, k, 0.5, A.data_ptr(), 71, B.data_ptr(), k,
                          -1.0, Cc.data_ptr(), m), (A, B, Cc)))
    c0s = [t[2].clone() for _, t in probs]
    with GroupedPlan([p for p, _ in probs]) as plan:
        for rep in range(2):
            if rep == 1:
                for _, (A, _, _) in probs:
                    A.mul_(-0.5).add_(0.25)
            for (_, t), c0 in zip(probs, c0s):
                t[2].copy_(c0)
            plan.launch()
            torch.cuda.synchronize()
            from_plan = [t[2].clone() for _, t in probs]
            for (_, t), c0 in zip(probs, c0s):
                t[2].copy_(c0)
            grouped_gemm([p for p, _ in probs])
            torch.cuda.synchronize()
            for i, ((p, t), fp) in enumerate(zip(probs, from_plan)):
                assert torch.equal(fp, t[2]), f"replay {rep} problem {i}"
    p, (A, B, Cc) = probs[-1]
    ref = restatement(p, A, B, c0s[-1])
    assert normwise(p, Cc.cpu().numpy(), ref, A, B, c0s[-1]) <= 4 * k * 2.0 ** -24


def test_server_result_same_alone_and_in_a_mix():
    rng = np.random.default_rng(61)
    target, (A, B, C0) = make_problem(rng, np.float64, Layout.RowMajor, 1, 0, 300, 257, 513, 1.25, -0.75)
    mix = random_mix(rng, 64)
    for grouped in (True, False):
        with Server(budget_bytes=256 << 20, max_batch=32, grouped=grouped) as srv:
            rid = srv.submit(target)
            st, d, ldd, t = srv.wait(rid)
            assert st == 0 and t[0] <= t[1] <= t[2]
            # the result is row-major m x n with leading dimension ldd
            alone_host = _read(d, target.m, target.n, ldd, np.float64, Layout.RowMajor)
            srv.release(rid)
            ids = []
            for i, (p, _) in enumerate(mix):
                ids.append((srv.submit(p), p))
                if i == 30:
                    rid = srv.submit(target)
            st, d, ldd, _ = srv.wait(rid)
            assert st == 0
            mixed_host = _read(d, target.m, target.n, ldd, np.float64, Layout.RowMajor)
            srv.release(rid)
            for r, p in ids:
                s2, _, _, _ = srv.wait(r)
                assert s2 == 0
                srv.release(r)
        assert np.array_equal(alone_host, mixed_host)
        ref = restatement(target, A, B, C0).reshape(target.m, target.n)
        den = 1.25 * float(A.norm()) * float(B.norm()) + 0.75 * float(C0.norm())
        assert np.linalg.norm(mixed_host - ref) / den <= 4 * 513 * 2.0 ** -53


def _read(ptr, m, n, ld, dt, layout):
    """Copy a server-owned result (raw device pointer) to a host m x n array."""
    rows, cols = (m, n) if layout == Layout.ColMajor else (n, m)

    class _View:
        __cuda_array_interface__ = {"shape": (ld * cols,), "typestr": np.dtype(dt).str,
                                    "data": (ptr, False), "version": 3}

    torch.cuda.synchronize()
    host = torch.as_tensor(_View(), device="cuda").cpu().numpy()
    mat = host.reshape(cols, ld)[:, :rows]
    return mat.T.copy() if layout == Layout.ColMajor else mat.copy()


def test_server_precision_forms_for_large_requests():
    """With set_forms, large requests run alone in the precision form (bit-
    identical to the single-call path in that form) while small ones stay on
    the grouped plain path; both in one serving run."""
    from rblas_b200.types import Precision
    rng = np.random.default_rng(66)
    bigs = [make_problem(rng, np.float32, Layout.RowMajor, 1, 0, 600, 500, 700, 1.5, -0.5),
            make_problem(rng, np.float64, Layout.ColMajor, 0, 1, 520, 610, 650, -0.75, 1.25),
            make_problem(rng, np.float64, Layout.RowMajor, 2, 2, 300, 900, 800, 0.5, 0.0)]
    small = random_mix(rng, 20, max_dim=200)
    for grouped in (True, False):
        with Server(budget_bytes=512 << 20, max_batch=32, grouped=grouped) as srv:
            srv.set_forms(Precision.Bf16x6, Precision.Ozaki, 1e8, 1e8)
            order = small[:10] + bigs + small[10:]
            ids = [srv.submit(p) for p, _ in order]
            got = []
            for rid, (p, _) in zip(ids, order):
                st, d, ldd, _ = srv.wait(rid)
                assert st == 0
                got.append(_read(d, p.m, p.n, ldd, p.dtype, p.layout))
                srv.release(rid)
        for (p, (A, B, C0)), g in zip(order, got):
            flop = 2.0 * p.m * p.n * p.k
            if flop >= 1e8:
                prec = Precision.Bf16x6 if p.dtype == np.float32 else Precision.Ozaki
                c = C0.clone()
                level3.gemm_dev(p.layout, p.transa, p.transb, p.m, p.n, p.k, p.alpha, p.a, p.lda, p.b, p.ldb,
                                p.beta, c.data_ptr(), p.ldc, p.dtype, prec=prec)
                torch.cuda.synchronize()
                h = c.cpu().numpy()
                exp = h.reshape(p.m, p.n) if p.layout == Layout.RowMajor else h.reshape(p.n, p.m).T
                assert np.array_equal(g, exp), (grouped, p.m, p.n, p.k)
            else:
                ref = restatement(p, A, B, C0)
                ref = ref.reshape(p.m, p.n) if p.layout == Layout.RowMajor else ref.reshape(p.n, p.m).T
                den = abs(p.alpha) * float(A.double().norm()) * float(B.double().norm()) + \
                    (abs(p.beta) * float(C0.double().norm()) if p.beta != 0.0 else 0.0)
                tol = 4 * max(p.k, 1) * (2.0 ** -24 if p.dtype == np.float32 else 2.0 ** -53)
                assert np.linalg.norm(g.astype(np.float64) - ref) / den <= tol


def test_server_budget_admission_and_busy():
    rng = np.random.default_rng(62)
    mix = random_mix(rng, 40, max_dim=300)
    # budget that holds only a few results at a time: requests wait for memory
    with Server(budget_bytes=2 << 20, max_batch=8, grouped=True) as srv:
        ids = [srv.submit(p) for p, _ in mix]
        for rid in ids:
            st, d, ldd, t = srv.wait(rid)
            assert st == 0
            srv.release(rid)
        big, _ = make_problem(rng, np.float64, Layout.ColMajor, 0, 0, 1024, 1024, 8, 1.0, 0.0)
        with pytest.raises(RuntimeError):
            srv.submit(big)  # 8 MiB result can never fit a 2 MiB budget


def test_server_trace_replay():
    rng = np.random.default_rng(63)
    mix = random_mix(rng, 120, max_dim=400)
    arrivals = np.cumsum(rng.exponential(1e9 / 20000, len(mix))).astype(np.uint64)
    for grouped in (True, False):
        with Server(budget_bytes=512 << 20, max_batch=64, grouped=grouped) as srv:
            st, times = srv.run_trace([p for p, _ in mix], arrivals)
        assert st == 0
        assert np.all(times[:, 0] <= times[:, 1]) and np.all(times[:, 1] <= times[:, 2])
        assert np.all(times[:, 2] > 0)
