"""Failure detection on the GPU without a fault: a bounded mbarrier wait that
cannot complete gives up after its time limit, the host reads the timeout
from the device error word, and the device keeps working."""
from __future__ import annotations

import ctypes as C
import time

import numpy as np
import pytest

import oracle
import rblas_b200 as rb
from rblas_b200 import _lib, level3
from rblas_b200.types import Layout, Transpose

RB_ERR_TIMEOUT = 8
RB_DEVERR_TIMEOUT = 0x01000000
PROBE_SITE = 0x7F0


@pytest.mark.gpu
def test_bounded_wait_gives_up_reports_and_leaves_the_device_usable():
    lib = _lib.load()
    detail = C.c_uint32(0)
    t0 = time.monotonic()
    st = lib.rb_probe_wait_timeout(C.byref(detail))
    dt = time.monotonic() - t0
    assert st == RB_ERR_TIMEOUT, (st, hex(detail.value))
    assert detail.value == RB_DEVERR_TIMEOUT | PROBE_SITE
    assert 1.9 <= dt < 60.0, dt  # gave up at its 2 s limit, not at once and not never
    assert rb.device_error() == (0, 0)  # the probe left the word clear
    # the next call runs normally: plain SGEMM within the parity bound of the restatement
    rng = np.random.default_rng(77)
    m, n, k = 96, 80, 130
    a = rng.uniform(-1, 1, m * k).astype(np.float32)
    b = rng.uniform(-1, 1, k * n).astype(np.float32)
    c0 = rng.uniform(-1, 1, m * n).astype(np.float32)
    c, ref = c0.copy(), c0.copy()
    level3.gemm(Layout.ColMajor, Transpose.NoTrans, Transpose.NoTrans, m, n, k, 1.5, a, m, b, k, -0.5, c, m)
    oracle.gemm(1, 0, 0, m, n, k, 1.5, a, m, b, k, -0.5, ref, m)
    d = c.astype(np.float64) - ref
    den = 1.5 * np.linalg.norm(a.astype(np.float64)) * np.linalg.norm(b.astype(np.float64)) + \
        0.5 * np.linalg.norm(c0.astype(np.float64))
    assert float(np.sqrt(np.sum(d * d)) / den) <= 4 * k * 2.0 ** -24
    assert rb.device_error() == (0, 0)
