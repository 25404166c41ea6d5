"""GPU tests of the autotuner (rb_autotune_*): it times every shape bucket --
the grouped plain kernel's split-K factor, and the Ozaki kernels' tile
width (128 x 256 or 128 x 128) -- writes a cache that loads back, the
planner follows the installed table, and results stay within the normwise
tolerance (4*k*u) of the restatement of rblas's gemm whatever factor the
table picks. The Ozaki tile width changes no result bit.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from rblas_b200 import level3
from rblas_b200.serving import (Problem, autotune, autotune_load, autotune_reset, grouped_gemm,
                                grouped_gemm_ozaki, grouped_splits)
from rblas_b200.types import Layout, Precision

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
    assert lines[0] == "rblas_b200 grouped autotune v2" and lines[1].startswith("device ")
    rows_all = [tuple(int(x) for x in ln.split()) for ln in lines[2:]]
    assert len(rows_all) == n
    rows = [r for r in rows_all if r[0] < 2]  # split factors
    widths = [r for r in rows_all if r[0] == 2]  # Ozaki tile widths
    assert rows and widths
    assert all(1 <= r[4] <= 16 for r in rows) and all(r[4] in (128, 256) for r in widths)
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
    # a width other than 128 or 256 is refused too
    bad.write_text(lines[0] + "\n" + lines[1] + "\n2 9 9 9 192\n")
    with pytest.raises(Exception):
        autotune_load(str(bad))


@pytest.mark.parametrize("width", [128, 256])
def test_ozaki_tile_width_changes_no_bit(tmp_path, width):
    """The same f64 problems in the Ozaki form, single calls and one grouped
    launch, with every bucket's tile width forced to 128 or 256 through a
    cache file: bit-identical to the built-in choice."""
    shapes = [(300, 200, 700), (513, 129, 1025), (700, 90, 300), (1000, 1000, 500)]
    probs = [_problem(np.float64, m, n, k, seed=80 + i) for i, (m, n, k) in enumerate(shapes)]
    autotune_reset()
    ref = []
    for p, A, B, C0 in probs:
        c = C0.clone()
        level3.gemm_dev(Layout.ColMajor, 0, 0, p.m, p.n, p.k, p.alpha, A.data_ptr(), p.m, B.data_ptr(), p.k,
                        p.beta, c.data_ptr(), p.m, np.float64, prec=Precision.Ozaki)
        ref.append(c)
    torch.cuda.synchronize()
    prop = torch.cuda.get_device_properties(0)
    lines = ["rblas_b200 grouped autotune v2",
             "device " + prop.name.replace(" ", "_") + " " + str(prop.multi_processor_count)]
    lines += [f"2 {lm} {ln} {lk} {width}" for lm in range(5, 13) for ln in range(5, 13) for lk in range(5, 13)]
    cache = tmp_path / "widths.txt"
    cache.write_text("\n".join(lines) + "\n")
    autotune_load(str(cache))
    try:
        for (p, A, B, C0), r in zip(probs, ref):
            c = C0.clone()
            level3.gemm_dev(Layout.ColMajor, 0, 0, p.m, p.n, p.k, p.alpha, A.data_ptr(), p.m, B.data_ptr(), p.k,
                            p.beta, c.data_ptr(), p.m, np.float64, prec=Precision.Ozaki)
            torch.cuda.synchronize()
            assert torch.equal(c, r), (p.m, p.n, p.k, width)
        outs = [C0.clone() for _, _, _, C0 in probs]
        qs = [Problem(np.float64, Layout.ColMajor, 0, 0, p.m, p.n, p.k, p.alpha, A.data_ptr(), p.m, B.data_ptr(),
                      p.k, p.beta, o.data_ptr(), p.m) for (p, A, B, _), o in zip(probs, outs)]
        grouped_gemm_ozaki(qs)
        torch.cuda.synchronize()
        for o, r in zip(outs, ref):
            assert torch.equal(o, r)
    finally:
        autotune_reset()


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
