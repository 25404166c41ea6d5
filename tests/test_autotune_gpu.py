"""GPU tests of the grouped kernel's split-K autotuner (rb_autotune_*): the
tuner times every shape bucket, writes a cache that loads back, the planner
follows the installed table, and results stay within the normwise tolerance
(4*k*u) of the restatement of rblas's gemm whatever factor the table picks.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from rblas_b200.serving import (Problem, autotune, autotune_load, autotune_reset, grouped_gemm,
                                grouped_splits)
from rblas_b200.types import Layout

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def tuned(tmp_path_factory):
    """Tune once for the module; the built-in rule is back afterwards."""
    cache = tmp_path_factory.mktemp("tune") / "grouped_splitk.txt"
    n = autotune(str(cache))
    yield cache, n
    autotune_reset()


def _problem(dt, m, n, k, seed):
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    tdt = torch.float32 if dt == np.float32 else torch.float64
    A = torch.randn(m * k, dtype=tdt, device="cuda", generator=g)
    B = torch.randn(k * n, dtype=tdt, device="cuda", generator=g)
    C0 = torch.randn(m * n, dtype=tdt, device="cuda", generator=g)
    p = Problem(dt, Layout.ColMajor, 0, 0, m, n, k, 1.25, A.data_ptr(), m, B.data_ptr(), k, -0.5,
                C0.data_ptr(), m)
    return p, A, B, C0


def test_autotune_writes_loadable_cache_and_planner_follows_it(tuned, tmp_path):
    cache, n = tuned
    assert n > 100
    lines = cache.read_text().splitlines()
    assert lines[0] == "rblas_b200 grouped split-k v1" and lines[1].startswith("device ")
    rows = [tuple(int(x) for x in ln.split()) for ln in lines[2:]]
    assert len(rows) == n and all(1 <= r[4] <= 16 for r in rows)
    autotune_reset()
    autotune_load(str(cache))
    # every tuned bucket's floor shape plans with the tuned factor
    # (clamped to the K-tiles the shape has)
    for dt, lm, ln, lk, s in rows[::7]:
        m, nn, k = 1 << lm, 1 << ln, 1 << lk
        bk = 32 if dt == 0 else 16
        p = Problem(np.float32 if dt == 0 else np.float64, Layout.ColMajor, 0, 0, m, nn, k, 1.0, 256, m,
                    256, k, 0.0, 256, m)
        num_kt = -(-k // bk)
        kps = -(-num_kt // min(s, num_kt))
        assert grouped_splits(p) == -(-num_kt // kps)
    # a corrupted cache is refused and leaves the loaded table in place
    bad = tmp_path / "bad.txt"
    bad.write_text("rblas_b200 grouped split-k v1\ndevice other 1\n")
    with pytest.raises(Exception):
        autotune_load(str(bad))


@pytest.mark.parametrize("dt,m,n,k", [(np.float32, 96, 200, 3500), (np.float64, 300, 100, 2900)])
def test_results_within_tolerance_under_tuned_table(tuned, dt, m, n, k):
    autotune_load(str(tuned[0]))
    p, A, B, C0 = _problem(dt, m, n, k, seed=70)
    c0 = C0.clone()
    grouped_gemm([p])
    torch.cuda.synchronize()
    c = c0.cpu().numpy().copy()
    oracle.gemm(int(Layout.ColMajor), 0, 0, m, n, k, 1.25, A.cpu().numpy(), m, B.cpu().numpy(), k, -0.5, c, m)
    d = C0.cpu().numpy().astype(np.float64) - c.astype(np.float64)
    den = 1.25 * float(A.double().norm()) * float(B.double().norm()) + 0.5 * float(c0.double().norm())
    u = 2.0 ** -24 if dt == np.float32 else 2.0 ** -53
    assert np.sqrt(np.sum(d * d)) / den <= 4 * k * u
