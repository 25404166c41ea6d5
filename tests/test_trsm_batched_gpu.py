"""GPU tests of the batched trsm (rb_?trsm_batched_dev) against the
restatement of rblas's trsm (src/level3.rs:390-520) run per batch member.

Well-conditioned triangular A (unit-range diagonal, small off-diagonal
entries, junk in the unreferenced triangle). Two bounds, u of the dtype:
the forward error against the oracle's solution, max-norm relative, within
1e3 * u (as the single-problem trsm tests), and the normwise backward error
of every member, ||op(A) X - alpha B||_F / (||A_tri||_F ||X||_F +
|alpha| ||B||_F) <= 4 * q * u (q the order of A) -- the bound of a blocked
substitution, which the f64 path's inverted diagonal blocks must also meet.
Covers every side/uplo/trans/diag, ragged sizes,
several right-hand-side slices per problem, the 16- and 8-wide slices of
large orders, padded leading dimensions and gaps between members (which must
stay untouched), unpadded even leading dimensions (the 16-byte operand
loads), and the leading-dimension errors.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from rblas_b200 import level3

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def tri(rng, q, uplo, dtype):
    off = rng.uniform(-0.1, 0.1, (q, q)) / max(1, q) ** 0.5
    A = np.tril(off, -1) if uplo == 1 else np.triu(off, 1)
    A = A + np.diag(rng.uniform(1, 2, q))
    junk = rng.uniform(-5, 5, (q, q))
    A = A + (np.triu(junk, 1) if uplo == 1 else np.tril(junk, -1))
    return np.asfortranarray(A.astype(dtype)).reshape(-1, order="F")


def _u(dtype):
    return 2.0 ** -24 if np.dtype(dtype) == np.float32 else 2.0 ** -53


def run_batch(rng, dtype, side, uplo, trans, diag, m, n, batch, alpha, pad=3, gap=(5, 7)):
    q = m if side == 0 else n
    lda, ldb = q + pad, m + pad
    sa, sb = lda * q + gap[0], ldb * n + gap[1]
    a_host = np.zeros(sa * batch, dtype=dtype)
    b_host = rng.uniform(-1, 1, sb * batch).astype(dtype)
    for i in range(batch):
        A = tri(rng, q, uplo, dtype).reshape(q, q, order="F")
        blk = a_host[i * sa:i * sa + lda * q].reshape(q, lda).T  # column-major view with lda
        blk[:q, :] = A
    tdt = torch.float32 if dtype == np.float32 else torch.float64
    A_d = torch.tensor(a_host, dtype=tdt, device="cuda")
    B_d = torch.tensor(b_host, dtype=tdt, device="cuda")
    level3.trsm_batched_dev(side, uplo, trans, diag, m, n, alpha, A_d.data_ptr(), lda, sa, B_d.data_ptr(), ldb, sb,
                            batch, dtype)
    torch.cuda.synchronize()
    got = B_d.cpu().numpy()
    worst = 0.0
    q_ord = m if side == 0 else n
    for i in range(batch):
        # backward error: op(A) X = alpha B (Left) or X op(A) = alpha B (Right)
        Am = a_host[i * sa:i * sa + lda * q_ord].reshape(q_ord, lda).T[:q_ord, :].astype(np.float64)
        T = np.tril(Am) if uplo == 1 else np.triu(Am)
        if diag == 1:
            np.fill_diagonal(T, 1.0)
        opA = T.T if trans else T
        X = got[i * sb:i * sb + ldb * n].reshape(n, ldb).T[:m, :].astype(np.float64)
        B0 = b_host[i * sb:i * sb + ldb * n].reshape(n, ldb).T[:m, :].astype(np.float64)
        R = (opA @ X if side == 0 else X @ opA) - alpha * B0
        den = np.linalg.norm(T) * np.linalg.norm(X) + abs(alpha) * np.linalg.norm(B0)
        back = np.linalg.norm(R) / den if den > 0 else np.linalg.norm(R)
        assert back <= 4 * q_ord * _u(dtype), (i, back, 4 * q_ord * _u(dtype))
        ref = b_host[i * sb:(i + 1) * sb].copy()
        oracle.trsm(side, uplo, trans, diag, m, n, alpha, np.ascontiguousarray(a_host[i * sa:(i + 1) * sa]), lda,
                    ref, ldb)
        g = got[i * sb:(i + 1) * sb]
        # inside each column: the m solved rows; the padding rows and the gap stay untouched
        sol = np.concatenate([ref[j * ldb:j * ldb + m] for j in range(n)])
        gs = np.concatenate([g[j * ldb:j * ldb + m] for j in range(n)])
        rel = np.max(np.abs(gs.astype(np.float64) - sol)) / max(np.max(np.abs(sol)), 1e-30)
        worst = max(worst, rel)
        untouched = np.ones(sb, dtype=bool)
        for j in range(n):
            untouched[j * ldb:j * ldb + m] = False
        assert np.array_equal(g[untouched], b_host[i * sb:(i + 1) * sb][untouched]), f"member {i} wrote outside B"
    return worst


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("side", [0, 1])
@pytest.mark.parametrize("uplo", [0, 1])
@pytest.mark.parametrize("trans", [0, 1])
def test_batched_trsm_parity(dtype, side, uplo, trans):
    rng = np.random.default_rng(80 + 8 * side + 4 * uplo + 2 * trans + (dtype == np.float64))
    for (m, n, batch) in [(1, 1, 3), (70, 33, 5), (150, 41, 4)]:
        for diag in (0, 1):
            rel = run_batch(rng, dtype, side, uplo, trans, diag, m, n, batch, 0.75)
            assert rel <= 1e3 * _u(dtype), ((m, n, batch), diag, rel)


def test_batched_trsm_config_shape_f64():
    """512 x 512 lower, 64 right-hand sides, f64 (four 16-wide slices on the
    FP64 tensor cores, two CTAs per SM)."""
    rng = np.random.default_rng(90)
    rel = run_batch(rng, np.float64, 0, 1, 0, 0, 512, 64, 6, 1.0)
    assert rel <= 1e3 * _u(np.float64)


def test_batched_trsm_wide_orders_use_narrow_slices():
    """Large orders: f64 q = 700 still fits two 16-wide slices per SM; q = 1400
    runs one 16-wide slice per SM (its q x 20 doubles of shared memory)."""
    rng = np.random.default_rng(91)
    for q, n in ((700, 20), (1400, 9)):
        rel = run_batch(rng, np.float64, 0, 0, 1, 0, q, n, 2, -1.5)
        assert rel <= 1e3 * _u(np.float64), (q, rel)


@pytest.mark.parametrize("side,q,nrhs,uplo,trans,diag,alpha", [
    (0, 512, 64, 1, 0, 0, 1.0),     # the config shape, Left Lower NoTrans: paired 16-byte A loads
    (0, 200, 40, 1, 0, 1, -0.75),   # ragged last diagonal block, Unit, three 16-wide slices
    (1, 256, 48, 1, 1, 0, 1.5),     # Right Lower Trans: the same loads, B read along its rows
    (0, 96, 17, 0, 1, 0, 2.0),      # Left Upper Trans: op(A)'s rows strided (element loads)
    (0, 700, 33, 1, 0, 0, 0.5),     # a large order: 16-wide slices, paired loads
])
def test_batched_trsm_aligned_operands_f64(side, q, nrhs, uplo, trans, diag, alpha):
    """Even leading dimensions and member strides on 16-byte-aligned
    operands: where op(A)'s rows are unit stride, adjacent A rows of a DMMA
    fragment load as one 16-byte pair. Gaps of 2 and 4 elements keep the
    strides even."""
    rng = np.random.default_rng(95 + q)
    m, n = (q, nrhs) if side == 0 else (nrhs, q)
    rel = run_batch(rng, np.float64, side, uplo, trans, diag, m, n, 3, alpha, pad=0, gap=(2, 4))
    assert rel <= 1e3 * _u(np.float64), (q, rel)


def test_batched_trsm_rejects_bad_leading_dims():
    from rblas_b200.error import InvalidLeadingDim
    A = torch.zeros(64, dtype=torch.float64, device="cuda")
    with pytest.raises(InvalidLeadingDim):
        level3.trsm_batched_dev(0, 1, 0, 0, 8, 4, 1.0, A.data_ptr(), 7, 64, A.data_ptr(), 8, 32, 1, np.float64)
    with pytest.raises(InvalidLeadingDim):
        level3.trsm_batched_dev(0, 1, 0, 0, 8, 4, 1.0, A.data_ptr(), 8, 64, A.data_ptr(), 7, 32, 1, np.float64)
