"""Benchmark of the GEMM engine on the DGEMM workload rblas's headline metric
is quoted on:

  f64, row-major, alpha=1.5, beta=-0.5, A/B/C0 i.i.d. standard normal (seeded):
  N/N, T/N, N/T, T/T at m=n=k=4096, plus N/N at m=3000 n=5000 k=2048.

One step = those five GEMMs (6.11e11 flop, counted as 2mnk). Inputs are
resident in HBM and larger than L2 (each 4096^2 f64 operand is 134 MB), so
no L2 flush is needed between steps.

  value    whole-job TFLOP/s, device-timed with CUDA events on the launching
           stream, inputs resident, max over ranks.
  e2e      the same step through the public host API (rb_dgemm_prec on pinned
           host buffers): every step copies A, B, C0 in and C out.
  forms    plain (FP64 on the CUDA cores) and, once built, the Ozaki INT8
           split-precision form, each timed the same way.
  roofline the dominant kernel against its pipe's measured peak.
  cpu_baseline  rblas's threaded gemm restated in C++ (the oracle), all host
           cores, on one step of this workload.

`--impl reference` times that CPU implementation alone on the same workload.
With torchrun (N > 1) every rank runs its own replica of the step (GEMM here
has no exchange step); value sums the work of all ranks over the max time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

ALPHA, BETA = 1.5, -0.5
BIG = 4096
EXTRA = (3000, 5000, 2048)
TRANS = [(0, 0), (1, 0), (0, 1), (1, 1)]  # (transa, transb): N/N, T/N, N/T, T/T


def step_gemms():
    """(ta, tb, m, n, k) of one step."""
    return [(ta, tb, BIG, BIG, BIG) for ta, tb in TRANS] + [(0, 0) + EXTRA]


def step_flops():
    return sum(2.0 * m * n * k for _, _, m, n, k in step_gemms())


def measured_peaks():
    """The pool's measured peaks (MEASURED_PEAKS.json beside this file), or None."""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return None


def dist_info():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Replicas:
    """One replica of the step per rank: GEMM has no exchange step, so the
    ranks share only the barrier before each timed region and the max over
    ranks of each time (every rank takes the same collective steps in the
    same order). `device` holds the reduction tensor: the rank's GPU for
    nccl, the CPU for gloo."""

    def __init__(self, backend, device):
        import torch
        self.torch = torch
        self.ws, self.rank, _ = dist_info()
        self.device = device
        self.dist = None
        if self.ws > 1:
            import torch.distributed as dist
            from datetime import timedelta
            dist.init_process_group(backend, timeout=timedelta(seconds=120))
            self.dist = dist

    def barrier(self):
        if self.dist:
            self.dist.barrier()

    def max(self, x):
        if not self.dist:
            return float(x)
        t = self.torch.tensor([float(x)], device=self.device, dtype=self.torch.float64)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    @staticmethod
    def value(work_per_rank, seconds, ws):
        """Whole-job throughput (TFLOP/s): every rank's work over the slowest rank's time."""
        return work_per_rank * ws / seconds / 1e12

    def close(self):
        if self.dist:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None


# --------------------------------------------------------------------------
# clocks
# --------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return None
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append(dict(sm=float(parts[1]), max=float(parts[2]), power=float(parts[3]),
                                 hw=parts[5], hwt=parts[6], swt=parts[7], swp=parts[8]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return None
        loaded = [r for r in rows if r["power"] > 250.0] or rows
        reasons = set()
        for r in loaded:
            if r["hw"] == "Active":
                reasons.add("hw_slowdown")
            if r["hwt"] == "Active":
                reasons.add("hw_thermal_slowdown")
            if r["swt"] == "Active":
                reasons.add("sw_thermal_slowdown")
            if r["swp"] == "Active":
                reasons.add("sw_power_cap")
        return {"sm_mhz": statistics.median(r["sm"] for r in loaded),
                "sm_max_mhz": max(r["max"] for r in rows), "reasons": sorted(reasons),
                "samples": len(rows), "samples_under_load": len(loaded)}


# --------------------------------------------------------------------------
# reference arm / CPU baseline: rblas's threaded gemm restated (the oracle)
# --------------------------------------------------------------------------

def make_host_operands(seed=1234):
    rng = np.random.default_rng(seed)
    ops = {}
    ops["A"] = rng.standard_normal(BIG * BIG)
    ops["B"] = rng.standard_normal(BIG * BIG)
    ops["C"] = rng.standard_normal(BIG * BIG)
    m, n, k = EXTRA
    ops["A2"] = rng.standard_normal(m * k)
    ops["B2"] = rng.standard_normal(k * n)
    ops["C2"] = rng.standard_normal(m * n)
    return ops


def cpu_step(ops, threads):
    import oracle
    for ta, tb, m, n, k in step_gemms():
        if m == BIG:
            a, b, c = ops["A"], ops["B"], ops["C"]
        else:
            a, b, c = ops["A2"], ops["B2"], ops["C2"]
        lda = m if ta else k          # row-major stored A: m x k (N) or k x m (T)
        ldb = k if tb else n
        oracle.gemm(0, ta, tb, m, n, k, ALPHA, a, lda, b, ldb, BETA, c, n, threads=threads)


def cpu_baseline(threads, reps=2):
    ops = make_host_operands()
    cpu_step(ops, threads)  # warm-up
    ts = []
    for _ in range(reps):
        t0 = time.perf_counter()
        cpu_step(ops, threads)
        ts.append(time.perf_counter() - t0)
    t = statistics.median(ts)
    return {"value": step_flops() / t / 1e12, "unit": "TFLOP/s", "cores": threads,
            "kind": "port",
            "sample": f"one full step (5 DGEMMs, {step_flops():.3e} flop), median of {reps} after "
                      f"1 warm-up; rblas threads-feature gemm restated in C++ (oracle/)"}


def level1_cpu_baseline(n=1 << 24, reps=3):
    """rblas's ddot and daxpy restated in C++ (oracle/: its AVX2 dot order and
    fused axpy), single thread as rblas's Level 1 is, on 2^24 f64 (128 MiB per
    vector, above the host caches), in the same bytes-per-call terms."""
    import oracle
    rng = np.random.default_rng(3)
    x = rng.standard_normal(n)
    y = rng.standard_normal(n)
    out = {"cores": 1, "kind": "port", "sample": f"n = {n} f64, median of {reps} after 1 warm-up"}
    for name, fn, nbytes in (("ddot", lambda: oracle.dot(n, x, 1, y, 1), 16.0 * n),
                             ("daxpy", lambda: oracle.axpy(n, 1e-3, x, 1, y, 1), 24.0 * n)):
        fn()
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            fn()
            ts.append(time.perf_counter() - t0)
        out[name + "_gb_s"] = nbytes / statistics.median(ts) / 1e9
    return out


def run_reference(args):
    ws, rank, _ = dist_info()
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    ops = make_host_operands()
    for _ in range(args.warmup):
        cpu_step(ops, threads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        cpu_step(ops, threads)
    dt = time.perf_counter() - t0
    value = step_flops() * args.steps / dt / 1e12
    line = {
        "impl": "reference", "metric": "DGEMM TFLOP/s (f64 row-major, 4 transposes @4096^3 + 3000x5000x2048)",
        "value": value, "unit": "TFLOP/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded normal)",
        "config": config_block(args),
        "cpu_baseline": {"value": value, "unit": "TFLOP/s", "cores": threads, "kind": "port",
                         "sample": "full steps of the workload on all host cores"},
        "e2e": {"value": value, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def config_block(args):
    return {"workload": "rblas DGEMM: f64 row-major alpha=1.5 beta=-0.5, N/N T/N N/T T/T at "
                        "4096^3 + N/N 3000x5000x2048",
            "gemms_per_step": 5, "flop_per_step": step_flops(), "l2": "inputs larger than L2",
            "parallelism": f"replicas x{args.gpus}"}


# --------------------------------------------------------------------------
# our arm
# --------------------------------------------------------------------------

def kernel_report():
    """Per-kernel {name: (launches, total_ms, total_work)} since the last call."""
    import ctypes as C

    from rblas_b200 import _lib
    buf = C.create_string_buffer(1 << 16)
    _lib.load().rb_kernel_timing_report(buf, len(buf))
    out = {}
    for line in buf.value.decode().splitlines():
        name, cnt, ms, work = line.split()
        out[name] = (int(cnt), float(ms), float(work))
    return out


def run_ours(args):
    import torch

    import rblas_b200 as rb
    from rblas_b200 import _lib, level3
    from rblas_b200.types import Layout, Precision

    ws, rank, local = dist_info()
    torch.cuda.set_device(local)
    rep = Replicas("nccl", torch.device("cuda", local))

    lib = rb.load_library()
    dev = torch.device("cuda", local)
    g = torch.Generator(device=dev)
    g.manual_seed(1234 + rank)
    A = torch.randn(BIG * BIG, dtype=torch.float64, device=dev, generator=g)
    B = torch.randn(BIG * BIG, dtype=torch.float64, device=dev, generator=g)
    Cs = [torch.randn(BIG * BIG, dtype=torch.float64, device=dev, generator=g) for _ in TRANS]
    m2, n2, k2 = EXTRA
    A2 = torch.randn(m2 * k2, dtype=torch.float64, device=dev, generator=g)
    B2 = torch.randn(k2 * n2, dtype=torch.float64, device=dev, generator=g)
    C2 = torch.randn(m2 * n2, dtype=torch.float64, device=dev, generator=g)
    stream = torch.cuda.current_stream(dev)
    sh = stream.cuda_stream

    def dev_step(prec):
        for i, (ta, tb, m, n, k) in enumerate(step_gemms()):
            if m == BIG:
                a, b, c = A, B, Cs[i]
            else:
                a, b, c = A2, B2, C2
            level3.gemm_dev(Layout.RowMajor, ta, tb, m, n, k, ALPHA, a.data_ptr(), m if ta else k,
                            b.data_ptr(), k if tb else n, BETA, c.data_ptr(), n, np.float64,
                            prec=prec, stream=sh)

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        rep.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        l0 = rb.launch_count()
        kernel_report()
        lib.rb_kernel_timing_enable(1)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        lib.rb_kernel_timing_enable(0)
        kr = kernel_report()
        launches = rb.launch_count() - l0
        ms = rep.max(e0.elapsed_time(e1))
        return ms / steps, launches, kr

    # ---- pipe peaks measured in this run (roofline denominators) ----------
    peaks = {"fp64_fma_tflops": float(lib.rb_probe_fma_peak_tflops(1, 0)),
             "fp32_fma_tflops": float(lib.rb_probe_fma_peak_tflops(0, 0)),
             "int8_tensor_tops": float(lib.rb_probe_tensor_peak_tflops(1, 0)),
             "bf16_tensor_tflops": float(lib.rb_probe_tensor_peak_tflops(0, 0))}

    forms = {}
    kreports = {}
    headline_name = "plain"
    clocks = None
    candidates = [("plain", Precision.Plain)]
    if args.form in ("auto", "ozaki"):
        candidates.append(("ozaki", Precision.Ozaki))
    for name, prec in candidates:
        try:
            dev_step(prec)
            torch.cuda.synchronize()
        except rb.BlasError as e:
            forms[name] = {"unavailable": str(e)}
            continue
        with ClockSampler(local) as cs:
            ms, launches, kr = timed(lambda: dev_step(prec), args.steps, args.warmup)
        forms[name] = {"tflops": Replicas.value(step_flops(), ms * 1e-3, ws), "ms_per_step": ms,
                       "gpu_launches": launches, "clocks": cs.summary()}
        kreports[name] = kr
        if name == "plain" or args.form != "plain":
            headline_name = name
            clocks = forms[name]["clocks"]
    hl = forms[headline_name]
    err_status = rb.device_error()

    # ---- roofline of the headline form's dominant kernel (live event timing)
    kr = kreports[headline_name]
    kname = max(kr, key=lambda n: kr[n][1])
    cnt, kms, work = kr[kname]
    achieved = work / (kms * 1e-3) / 1e12
    if kname.startswith("umma_ozaki"):
        peak, unit, bound = peaks["int8_tensor_tops"], "TOP/s", "tensor"
        psrc = "INT8 tcgen05 throughput measured in-run by rb_probe_tensor_peak_tflops (back-to-back M128 N256 K32 UMMAs, smem operands); not in MEASURED_PEAKS.json"
    else:
        peak, unit, bound = peaks["fp64_fma_tflops"], "TFLOP/s", "fp64"
        psrc = ("FP64 throughput measured in-run by rb_probe_fma_peak_tflops (DFMA; the plain DGEMM runs on DMMA, "
                "whose peak on this GPU measured the same, 36.8-37.0 TFLOP/s); not in MEASURED_PEAKS.json")
    # DRAM bytes per launch of the dominant kernel, measured by ncu
    # (dram__bytes_read.sum + dram__bytes_write.sum) on one launch of each of
    # the step's shapes: 2.186 GB at 4096^3 (x4 per step), 1.067 GB at
    # 3000x5000x2048 (x1)
    traffic = (4 * 2.186e9 + 1.067e9) / 5 if kname == "umma_ozaki_i8" else None
    # second denominator for the INT8 pipe: twice the driver-measured dense
    # BF16 cuBLAS burst (the INT8 tensor rate is twice the BF16 rate)
    mp = measured_peaks() or {}
    alt = 2.0 * mp["bf16_tflops"] if (kname.startswith("umma_ozaki") and mp.get("bf16_tflops")) else None
    roofline = {"bound": bound, "achieved": achieved, "peak": peak, "unit": unit,
                "frac": achieved / peak if peak > 0 else None,
                "peak_alt": alt, "frac_alt": achieved / alt if alt else None,
                "peak_alt_source": "2 x MEASURED_PEAKS.json bf16_tflops (burst)" if alt else None,
                "traffic": traffic,
                "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum per launch, averaged over "
                                   "the step's launch shapes") if traffic else None,
                "kernel": kname, "launches": cnt, "avg_launch_ms": kms / cnt,
                "work_per_launch": work / cnt, "peak_source": psrc,
                "kernels": {k: {"launches": v[0], "ms": v[1]} for k, v in kr.items()}}

    # ---- SGEMM 8192^3 col-major alpha=1 beta=1: plain vs BF16 split forms
    sgemm = {}
    if not args.no_sgemm:
        n8 = 8192
        gs = torch.Generator(device=dev)
        gs.manual_seed(77)
        SA = torch.rand(n8 * n8, dtype=torch.float32, device=dev, generator=gs) * 2 - 1
        SB = torch.rand(n8 * n8, dtype=torch.float32, device=dev, generator=gs) * 2 - 1
        SC = torch.rand(n8 * n8, dtype=torch.float32, device=dev, generator=gs) * 2 - 1
        for name, prec, reps in (("plain", Precision.Plain, 3), ("bf16x3", Precision.Bf16x3, 5),
                                 ("bf16x6", Precision.Bf16x6, 5)):
            def one():
                level3.gemm_dev(Layout.ColMajor, 0, 0, n8, n8, n8, 1.0, SA.data_ptr(), n8, SB.data_ptr(),
                                n8, 1.0, SC.data_ptr(), n8, np.float32, prec=prec, stream=sh)
            ms, launches, kr2 = timed(one, reps, 2)
            sgemm[name] = {"tflops": 2.0 * n8 ** 3 / (ms * 1e-3) / 1e12, "ms": ms,
                           "kernels": {k: {"launches": v[0], "ms": v[1],
                                           "pipe_tflops": v[2] / (v[1] * 1e-3) / 1e12}
                                       for k, v in kr2.items()}}
        del SA, SB, SC
        torch.cuda.empty_cache()

    # ---- DGEMM 8192^3 row-major N/N alpha=1.5 beta=-0.5: plain (DMMA) vs Ozaki
    dgemm8 = {}
    if not args.no_sgemm:
        n8 = 8192
        gd = torch.Generator(device=dev)
        gd.manual_seed(78)
        DA = torch.randn(n8 * n8, dtype=torch.float64, device=dev, generator=gd)
        DB = torch.randn(n8 * n8, dtype=torch.float64, device=dev, generator=gd)
        DC = torch.randn(n8 * n8, dtype=torch.float64, device=dev, generator=gd)
        for name, prec, reps in (("plain", Precision.Plain, 3), ("ozaki", Precision.Ozaki, 5)):
            def one():
                level3.gemm_dev(Layout.RowMajor, 0, 0, n8, n8, n8, ALPHA, DA.data_ptr(), n8, DB.data_ptr(),
                                n8, BETA, DC.data_ptr(), n8, np.float64, prec=prec, stream=sh)
            ms, launches, kr2 = timed(one, reps, 2)
            dgemm8[name] = {"tflops": 2.0 * n8 ** 3 / (ms * 1e-3) / 1e12, "ms": ms,
                            "kernels": {k: {"launches": v[0], "ms": v[1],
                                            "pipe_tflops": v[2] / (v[1] * 1e-3) / 1e12}
                                        for k, v in kr2.items()}}
        if "plain" in dgemm8 and "ozaki" in dgemm8:
            dgemm8["ozaki_over_plain"] = dgemm8["ozaki"]["tflops"] / dgemm8["plain"]["tflops"]
        del DA, DB, DC
        torch.cuda.empty_cache()

    # ---- the other configurations: SGEMM 1024^3 (C1), tall-skinny SGEMM
    # 65536x128x8192 (C3), complex 2048^3 ConjTrans/NoTrans (C4) and the
    # batched f64 trsm 512^2 x 64 right-hand sides x 1024 (C4)
    others = {}
    if not args.no_configs:
        from rblas_b200 import complex3

        # the configurations are measured from an idle GPU: right after the
        # 8192^3 Ozaki runs above, a 1024^3 SGEMM ran 15-25 % slower for about
        # two seconds (SM clock unchanged), then recovered
        if not args.no_sgemm:
            torch.cuda.synchronize()
            time.sleep(2.0)

        def form_times(fn_for, work, forms, reps):
            res = {}
            for name, prec in forms:
                ms, launches, kr3 = timed(fn_for(prec), reps, 2)
                res[name] = {"tflops": work / (ms * 1e-3) / 1e12, "ms": ms, "launches_per_call": launches / reps,
                             "kernels": {k: {"launches": v[0], "ms": v[1]} for k, v in kr3.items()}}
            return res

        g2 = torch.Generator(device=dev)
        g2.manual_seed(1234)
        # C1: f32 col-major NN 1024^3, alpha = 1, beta = 0
        n1 = 1024
        X1 = [torch.rand(n1 * n1, dtype=torch.float32, device=dev, generator=g2) * 2 - 1 for _ in range(3)]
        others["c1_sgemm_1024"] = form_times(
            lambda prec: (lambda: level3.gemm_dev(Layout.ColMajor, 0, 0, n1, n1, n1, 1.0, X1[0].data_ptr(), n1,
                                                  X1[1].data_ptr(), n1, 0.0, X1[2].data_ptr(), n1, np.float32,
                                                  prec=prec, stream=sh)),
            2.0 * n1 ** 3, (("plain", Precision.Plain), ("bf16x3", Precision.Bf16x3), ("bf16x6", Precision.Bf16x6)), 20)
        del X1
        # C3 tall-skinny: 65536 x 128 x 8192, alpha = beta = 1
        m3, n3, k3 = 65536, 128, 8192
        A3 = torch.rand(m3 * k3, dtype=torch.float32, device=dev, generator=g2) * 2 - 1
        B3 = torch.rand(k3 * n3, dtype=torch.float32, device=dev, generator=g2) * 2 - 1
        C3 = torch.rand(m3 * n3, dtype=torch.float32, device=dev, generator=g2) * 2 - 1
        others["c3_sgemm_65536x128x8192"] = form_times(
            lambda prec: (lambda: level3.gemm_dev(Layout.ColMajor, 0, 0, m3, n3, k3, 1.0, A3.data_ptr(), m3,
                                                  B3.data_ptr(), k3, 1.0, C3.data_ptr(), m3, np.float32,
                                                  prec=prec, stream=sh)),
            2.0 * m3 * n3 * k3, (("plain", Precision.Plain), ("bf16x3", Precision.Bf16x3), ("bf16x6", Precision.Bf16x6)), 5)
        c3 = others["c3_sgemm_65536x128x8192"]
        c3["min_bytes"] = 4 * (m3 * k3 + k3 * n3 + 2 * m3 * n3)
        # near the HBM ridge: the minimum bytes (A, B once, C read and written) over each form's time
        for form in ("plain", "bf16x3", "bf16x6"):
            c3[form]["min_bytes_gbs"] = c3["min_bytes"] / (c3[form]["ms"] * 1e-3) / 1e9
        del A3, B3, C3
        # C4 complex: ConjTrans/NoTrans 2048^3, alpha = (1, 0.5), beta = 0; 8mnk real flop (4M)
        n4 = 2048
        for cdt, tdt, cforms in ((np.complex128, torch.float64, (("plain", Precision.Plain), ("ozaki", Precision.Ozaki))),
                                 (np.complex64, torch.float32, (("plain", Precision.Plain), ("bf16x3", Precision.Bf16x3),
                                                                ("bf16x6", Precision.Bf16x6)))):
            Xc = [torch.randn(2 * n4 * n4, dtype=tdt, device=dev, generator=g2) for _ in range(3)]
            others["c4_%s_2048_CN" % ("zgemm" if cdt == np.complex128 else "cgemm")] = form_times(
                lambda prec: (lambda: complex3.gemm_dev(2, 0, n4, n4, n4, 1.0 + 0.5j, Xc[0].data_ptr(), n4,
                                                        Xc[1].data_ptr(), n4, 0.0, Xc[2].data_ptr(), n4, cdt,
                                                        prec=prec, stream=sh)),
                8.0 * n4 ** 3, cforms, 4)
            del Xc
        # C4 batched trsm: 1024 x (512 x 512 lower, 64 RHS), f64; m^2 n flop each
        qb, nb_, batch = 512, 64, 1024
        At = torch.randn(qb * qb * batch, dtype=torch.float64, device=dev, generator=g2) * (0.1 / qb ** 0.5)
        At.view(batch, qb, qb).diagonal(dim1=1, dim2=2).uniform_(1.0, 2.0)
        Bt = torch.rand(qb * nb_ * batch, dtype=torch.float64, device=dev, generator=g2) * 2 - 1
        ms, launches, kr4 = timed(lambda: level3.trsm_batched_dev(0, 1, 0, 0, qb, nb_, 1.0, At.data_ptr(), qb,
                                                                  qb * qb, Bt.data_ptr(), qb, qb * nb_, batch,
                                                                  np.float64, stream=sh), 5, 2)
        others["c4_dtrsm_batched_512x64x1024"] = {
            "tflops": qb * qb * nb_ * batch / (ms * 1e-3) / 1e12, "ms": ms, "launches_per_call": launches / 5,
            "kernels": {k: {"launches": v[0], "ms": v[1]} for k, v in kr4.items()}}
        del At, Bt
        torch.cuda.empty_cache()
        # Level 2 (HBM-bound): dgemv 16384^2 col-major N and T (m*n*8 bytes of
        # A per call), dger 16384^2 (A read and written: 2*m*n*8 bytes)
        from rblas_b200 import level2
        n2l = 16384
        AL = torch.randn(n2l * n2l, dtype=torch.float64, device=dev, generator=g2)
        xl = torch.randn(n2l, dtype=torch.float64, device=dev, generator=g2)
        yl = torch.randn(n2l, dtype=torch.float64, device=dev, generator=g2)
        hbm = (measured_peaks() or {}).get("hbm_gbs")
        lv2 = {"hbm_peak_gbs": hbm, "peak_source": "MEASURED_PEAKS.json hbm_gbs" if hbm else None}
        for name, fn, nbytes in (
                ("dgemv_N", lambda: level2.gemv_dev(1, 0, n2l, n2l, 1.0, AL.data_ptr(), n2l, xl.data_ptr(), 1, 0.5,
                                                    yl.data_ptr(), 1, np.float64, stream=sh), 8.0 * n2l * n2l),
                ("dgemv_T", lambda: level2.gemv_dev(1, 1, n2l, n2l, 1.0, AL.data_ptr(), n2l, xl.data_ptr(), 1, 0.5,
                                                    yl.data_ptr(), 1, np.float64, stream=sh), 8.0 * n2l * n2l),
                ("dger", lambda: level2.ger_dev(1, n2l, n2l, 1e-3, xl.data_ptr(), 1, yl.data_ptr(), 1, AL.data_ptr(),
                                                n2l, np.float64, stream=sh), 16.0 * n2l * n2l)):
            ms, launches, _ = timed(fn, 10, 2)
            gbs = nbytes / (ms * 1e-3) / 1e9
            lv2[name] = {"ms": ms, "gb_s": gbs, "frac_of_hbm": gbs / hbm if hbm else None,
                         "launches_per_call": launches / 10}
        others["level2_16384"] = lv2
        del AL, xl, yl
        torch.cuda.empty_cache()
        # Level 1 (HBM-bound): 2^27 f64 per vector (1 GiB each, above L2, so
        # every call streams from HBM); f32 and complex forms over the same bytes
        n1 = 1 << 27
        keep1, cases1 = level1_cases(torch, n1, dev, sh)
        lv1 = {"hbm_peak_gbs": hbm, "peak_source": "MEASURED_PEAKS.json hbm_gbs" if hbm else None,
               "vector_bytes": 8 * n1}
        for name, fn, nbytes in cases1:
            ms, launches, _ = timed(fn, 10, 3)
            gbs = nbytes / (ms * 1e-3) / 1e9
            lv1[name] = {"ms": ms, "gb_s": gbs, "frac_of_hbm": gbs / hbm if hbm else None,
                         "launches_per_call": launches / 10}
        # launch-bound end: rblas's own bench sizes (1M f32, src benches/level1.rs)
        small = torch.ones(2 << 20, dtype=torch.float32, device=dev)
        from rblas_b200 import level1 as l1mod
        for name, fn in (("saxpy_1M_us", lambda: l1mod.axpy_dev(1 << 20, 3.0, small.data_ptr(), 1,
                                                                  small[1 << 20:].data_ptr(), 1, np.float32, sh)),
                         ("sdot_1M_us", lambda: l1mod.dot_dev(1 << 20, small.data_ptr(), 1, small[1 << 20:].data_ptr(),
                                                              1, keep1[2].data_ptr(), np.float32, sh))):
            ms, _, _ = timed(fn, 200, 20)
            lv1[name] = ms * 1e3
        if rank == 0 and ws == 1 and not args.no_cpu:
            lv1["cpu_baseline"] = level1_cpu_baseline()
        others["level1_2^27_f64"] = lv1
        del keep1, cases1, small
        torch.cuda.empty_cache()

    # ---- e2e through the public host API (pinned host buffers) -------------
    e2e = None
    if not args.no_e2e:
        def pinned(n, src):
            t = torch.empty(n, dtype=torch.float64, pin_memory=True)
            t.copy_(src.cpu())
            return t
        hA, hB = pinned(BIG * BIG, A), pinned(BIG * BIG, B)
        hC = [pinned(BIG * BIG, c) for c in Cs]
        hA2, hB2, hC2 = pinned(m2 * k2, A2), pinned(k2 * n2, B2), pinned(m2 * n2, C2)
        prec = Precision.Ozaki if headline_name == "ozaki" else Precision.Plain

        def host_step():
            h2d = d2h = 0
            for i, (ta, tb, m, n, k) in enumerate(step_gemms()):
                if m == BIG:
                    a, b, c = hA.numpy(), hB.numpy(), hC[i].numpy()
                else:
                    a, b, c = hA2.numpy(), hB2.numpy(), hC2.numpy()
                level3.gemm(Layout.RowMajor, ta, tb, m, n, k, ALPHA, a, m if ta else k, b,
                            k if tb else n, BETA, c, n, prec=prec)
                h2d += (a.nbytes + b.nbytes + c.nbytes)
                d2h += c.nbytes
            return h2d, d2h

        for _ in range(max(1, args.warmup)):
            host_step()
        rep.barrier()
        torch.cuda.synchronize()
        k_e2e = max(2, args.steps // 2)
        t0 = time.perf_counter()
        for _ in range(k_e2e):
            h2d, d2h = host_step()
        torch.cuda.synchronize()
        dt = rep.max((time.perf_counter() - t0) / k_e2e)
        e2e = {"value": Replicas.value(step_flops(), dt, ws), "unit": "TFLOP/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "steps": k_e2e,
               "timing": "host wall clock around synchronous host-API calls (pinned buffers)"}

    # ---- serving: a 5000-request slice of the request stream (the full
    # 20,000-request sweep is `--serve`), grouped vs per-request launches
    serving = None
    if not args.no_serve and rank == 0 and ws == 1:
        from rblas_b200.serving import autotune
        tuned = autotune()
        serving = run_serving(torch, [10000.0, 15000.0, 20000.0, 25000.0, 30000.0, 50000.0], 5000, 60 << 30)
        serving["autotuned_buckets"] = tuned
        serving["note"] = ("5000-request slice of the serving stream; operands resident in HBM; "
                           "latency = enqueue -> completion observed by the server")

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cpu = cpu_baseline(os.cpu_count() or 1)

    if rank == 0:
        line = {
            "metric": "DGEMM TFLOP/s (f64 row-major, 4 transposes @4096^3 + 3000x5000x2048)",
            "value": hl["tflops"], "unit": "TFLOP/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": hl["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded standard normal, generated on device)",
            "form": headline_name, "config": config_block(args), "forms": forms,
            "clocks": clocks, "e2e": e2e, "gpu_launches": hl["gpu_launches"],
            "roofline": roofline, "cpu_baseline": cpu, "peaks_measured": peaks,
            "sgemm_8192": sgemm, "dgemm_8192": dgemm8, "configs": others, "serving": serving,
            "device_error": {"after_headline": err_status[0], "end_of_run": rb.device_error()[0]},
        }
        print(json.dumps(line))
    rep.close()


# --------------------------------------------------------------------------
# serving: the request stream of the serving configuration
# --------------------------------------------------------------------------

def serving_trace(n_req, seed=5):
    """Request shapes of the serving configuration: m, n, k log-uniform in
    [32, 4096], dtype 50/50 f32/f64, layout and transposes uniform, alpha and
    beta uniform in [-2, 2]."""
    rng = np.random.default_rng(seed)
    lo, hi = np.log(32), np.log(4096)
    mnk = np.exp(rng.uniform(lo, hi, (n_req, 3))).astype(np.int64)
    return dict(mnk=mnk, dtype=rng.integers(0, 2, n_req), layout=rng.integers(0, 2, n_req),
                ta=rng.integers(0, 3, n_req), tb=rng.integers(0, 3, n_req),
                alpha=rng.uniform(-2, 2, n_req), beta=rng.uniform(-2, 2, n_req),
                offs=rng.integers(0, 1 << 20, (n_req, 3)))


# precision forms for large serving requests (each within 2x of plain's
# error against the FP64 oracle): f32 >= 2e8 flop in BF16X6, f64 >= 1e9 flop
# in Ozaki; smaller requests stay on the grouped plain kernel
SERVE_FORMS = {"f32_form": 3, "f64_form": 2, "f32_min_flop": 2e8, "f64_min_flop": 1e9}


def run_serving(torch, rates, n_req, budget, max_batch=256, seed=5, with_forms=True):
    """Replay a Poisson stream of n_req requests at each rate through the
    server in grouped mode and in per-request mode. Operands are standard
    normal values resident in HBM (pools the requests point into)."""
    from rblas_b200.serving import Problem, Server

    tr = serving_trace(n_req, seed)
    big = 4096 * 4096
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    pools = {0: torch.randn(big + (1 << 22), dtype=torch.float32, device="cuda", generator=g),
             1: torch.randn(big + (1 << 22), dtype=torch.float64, device="cuda", generator=g)}
    problems, flops = [], 0.0
    for i in range(n_req):
        m, n, k = (int(x) for x in tr["mnk"][i])
        dt = int(tr["dtype"][i])
        vec = 4 if dt == 0 else 2
        layout, ta, tb = int(tr["layout"][i]), int(tr["ta"][i]), int(tr["tb"][i])
        ar, ac = (k, m) if ta else (m, k)
        br, bc = (n, k) if tb else (k, n)
        pad = lambda x: (x + vec - 1) // vec * vec
        lda = pad(ar) if layout == 1 else pad(ac)
        ldb = pad(br) if layout == 1 else pad(bc)
        ldc = pad(m) if layout == 1 else pad(n)
        base = pools[dt].data_ptr()
        es = 4 if dt == 0 else 8
        offs = [int(o) // 16 * 16 for o in tr["offs"][i]]  # 16-element aligned
        problems.append(Problem(np.float32 if dt == 0 else np.float64, layout, ta, tb, m, n, k,
                                float(tr["alpha"][i]), base + offs[0] * es, lda, base + offs[1] * es, ldb,
                                float(tr["beta"][i]), base + offs[2] * es, ldc))
        flops += 2.0 * m * n * k
    out = {"requests": n_req, "flop": flops, "budget_bytes": budget, "max_batch": max_batch, "rates": []}
    rng = np.random.default_rng(seed + 1)
    gaps = rng.exponential(1.0, n_req)
    for rate in rates:
        arrivals = (np.cumsum(gaps) / rate * 1e9).astype(np.uint64)
        row = {"rate_req_s": rate}
        modes = [("grouped", True, False), ("per_request", False, False)]
        if with_forms:
            modes += [("grouped_forms", True, True), ("per_request_forms", False, True)]
        for mode, grouped, forms in modes:
            # all modes admit the same sets; per-request mode launches the
            # single-problem plain kernel once per request, grouped mode one
            # grouped plain launch per set, grouped_forms runs the large
            # requests of each set in the precision forms (the f64 ones in one
            # grouped Ozaki launch, the f32 ones in one grouped BF16X6
            # launch), per_request_forms the same arithmetic with one launch
            # per request
            with Server(budget_bytes=budget, max_batch=max_batch, grouped=grouped) as srv:
                if forms:
                    srv.set_forms(**SERVE_FORMS)
                st, times = srv.run_trace(problems, arrivals)
            lat = (times[:, 2].astype(np.int64) - times[:, 0].astype(np.int64)) / 1e6
            span = (int(times[:, 2].max()) - int(times[:, 0].min())) / 1e9
            row[mode] = {"status": int(st), "tflops": flops / span / 1e12, "span_s": span,
                         "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99))}
        out["rates"].append(row)
    # throughput at equal p99: for each latency bound, the highest aggregate
    # TFLOP/s each mode sustained with p99 within it (None: no rate met it)
    slo = []
    for bound in (2.0, 5.0, 10.0, 20.0, 50.0, 100.0):
        best = {}
        for mode in ("grouped", "per_request", "grouped_forms", "per_request_forms"):
            ok = [r[mode]["tflops"] for r in out["rates"] if mode in r and r[mode]["p99_ms"] <= bound]
            best[mode] = max(ok) if ok else None
        pr, prf = best["per_request"], best["per_request_forms"]
        slo.append({"p99_bound_ms": bound, "grouped_tflops": best["grouped"], "per_request_tflops": pr,
                    "grouped_forms_tflops": best["grouped_forms"], "per_request_forms_tflops": prf,
                    "ratio": (best["grouped"] / pr) if best["grouped"] and pr else None,
                    "ratio_forms": (best["grouped_forms"] / pr) if best["grouped_forms"] and pr else None,
                    "ratio_forms_same_arith": (best["grouped_forms"] / prf) if best["grouped_forms"] and prf
                    else None})
    out["at_equal_p99"] = slo
    if with_forms:
        out["forms"] = dict(SERVE_FORMS, note="grouped_forms: the requests of a set at or above the flop "
                                              "thresholds run in one grouped BF16X6 launch (f32) and one grouped "
                                              "Ozaki launch (f64), the rest in one grouped plain launch; "
                                              "per_request_forms: the same forms, one launch per request")
    sat = max(out["rates"], key=lambda r: r["rate_req_s"])
    out["saturated"] = {"rate_req_s": sat["rate_req_s"], "grouped_tflops": sat["grouped"]["tflops"],
                        "per_request_tflops": sat["per_request"]["tflops"],
                        "ratio": sat["grouped"]["tflops"] / sat["per_request"]["tflops"]}
    if with_forms:
        out["saturated"]["grouped_forms_tflops"] = sat["grouped_forms"]["tflops"]
        out["saturated"]["per_request_forms_tflops"] = sat["per_request_forms"]["tflops"]
        out["saturated"]["ratio_forms"] = sat["grouped_forms"]["tflops"] / sat["per_request"]["tflops"]
        out["saturated"]["ratio_forms_same_arith"] = (sat["grouped_forms"]["tflops"] /
                                                      sat["per_request_forms"]["tflops"])
    del pools
    torch.cuda.empty_cache()
    return out


def run_serve_mode(args):
    import torch
    torch.cuda.set_device(0)
    if args.serve_thresholds:
        f32_min, f64_min = (float(x) for x in args.serve_thresholds.split(","))
        SERVE_FORMS.update(f32_min_flop=f32_min, f64_min_flop=f64_min)
    if not args.no_autotune:
        from rblas_b200.serving import autotune
        autotune()
    rates = [float(r) for r in args.rates.split(",")]
    res = run_serving(torch, rates, args.requests, int(args.budget_gb * (1 << 30)))
    print(json.dumps({"serving": res}))


def run_kernel_only(args):
    """One GEMM shape, launched warmup + steps times on the device (for ncu
    captures of a single kernel on a bounded case)."""
    import torch

    from rblas_b200 import level3
    from rblas_b200.types import Layout, Precision

    m, n, k = args.shape
    dt = torch.float64 if args.dtype == "f64" else torch.float32
    g = torch.Generator(device="cuda")
    g.manual_seed(7)
    A = torch.randn(m * k, dtype=dt, device="cuda", generator=g)
    B = torch.randn(k * n, dtype=dt, device="cuda", generator=g)
    C = torch.randn(m * n, dtype=dt, device="cuda", generator=g)
    prec = {"plain": Precision.Plain, "ozaki": Precision.Ozaki, "bf16x3": Precision.Bf16x3,
            "bf16x6": Precision.Bf16x6}[args.form if args.form != "auto" else "plain"]
    sh = torch.cuda.current_stream().cuda_stream
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    for i in range(args.warmup + args.steps):
        if i == args.warmup:
            e0.record()
        level3.gemm_dev(Layout.ColMajor, args.ta, args.tb, m, n, k, 1.0, A.data_ptr(),
                        k if args.ta else m, B.data_ptr(), n if args.tb else k, 0.5, C.data_ptr(), m,
                        np.float64 if args.dtype == "f64" else np.float32, prec=prec, stream=sh)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / max(args.steps, 1)
    print(json.dumps({"kernel_only": [m, n, k], "dtype": args.dtype, "form": args.form,
                      "ms": ms, "tflops": 2.0 * m * n * k / (ms * 1e-3) / 1e12}))


def level1_cases(torch, n, dev, sh, seed=11):
    """Level-1 calls on device vectors of n scalars (f64 / f32 views of the
    same 8n-byte buffers; complex over n/2 elements), each with its
    algorithmic HBM bytes per call: axpy reads x, y and writes y (3 vectors),
    dot reads 2, asum / nrm2 read 1, scal reads and writes 1, copy reads 1 and
    writes 1, swap reads and writes 2."""
    from rblas_b200 import complex1, level1
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    x = torch.randn(n, dtype=torch.float64, device=dev, generator=g)
    y = torch.randn(n, dtype=torch.float64, device=dev, generator=g)
    r = torch.zeros(4, dtype=torch.float64, device=dev)
    xs, ys = x.view(torch.float32), y.view(torch.float32)  # 2n f32 over the same bytes
    px, py, pr, B = x.data_ptr(), y.data_ptr(), r.data_ptr(), 8.0 * n
    f64, f32, c128 = np.float64, np.float32, np.complex128
    return (x, y, r), [
        ("daxpy", lambda: level1.axpy_dev(n, 1e-3, px, 1, py, 1, f64, sh), 3 * B),
        ("ddot", lambda: level1.dot_dev(n, px, 1, py, 1, pr, f64, sh), 2 * B),
        ("dnrm2", lambda: level1.nrm2_dev(n, px, 1, pr, f64, sh), B),
        ("dasum", lambda: level1.asum_dev(n, px, 1, pr, f64, sh), B),
        ("dscal", lambda: level1.scal_dev(n, 1.0 - 1e-9, py, 1, f64, sh), 2 * B),
        ("dcopy", lambda: level1.copy_dev(n, px, 1, py, 1, f64, sh), 2 * B),
        ("dswap", lambda: level1.swap_dev(n, px, 1, py, 1, f64, sh), 4 * B),
        ("saxpy", lambda: level1.axpy_dev(2 * n, 1e-3, xs.data_ptr(), 1, ys.data_ptr(), 1, f32, sh), 3 * B),
        ("sdot", lambda: level1.dot_dev(2 * n, xs.data_ptr(), 1, ys.data_ptr(), 1, pr, f32, sh), 2 * B),
        ("snrm2", lambda: level1.nrm2_dev(2 * n, xs.data_ptr(), 1, pr, f32, sh), B),
        ("zaxpy", lambda: complex1.axpy_dev(n // 2, 1e-3 + 1e-3j, px, 1, py, 1, c128, sh), 3 * B),
        ("zdotc", lambda: complex1.dotc_dev(n // 2, px, 1, py, 1, pr, c128, sh), 2 * B),
        ("dznrm2", lambda: complex1.nrm2_dev(n // 2, px, 1, pr, c128, sh), B),
        ("daxpy_incx2", lambda: level1.axpy_dev(n // 2, 1e-3, px, 2, py, 2, f64, sh), 3 * B / 2),
    ]


def run_level1_only(args):
    """The Level-1 calls of `level1_cases` on n-scalar f64 vectors, each
    launched warmup + steps times (for ncu captures on a bounded case)."""
    import torch

    n = args.level1
    sh = torch.cuda.current_stream().cuda_stream
    keep, cases = level1_cases(torch, n, "cuda", sh)
    out = {"level1": n}
    for name, fn, nbytes in cases:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        for i in range(args.warmup + args.steps):
            if i == args.warmup:
                e0.record()
            fn()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / max(args.steps, 1)
        out[name] = {"ms": ms, "gb_s": nbytes / (ms * 1e-3) / 1e9}
    print(json.dumps(out))


def run_level2_only(args):
    """dgemv (N and T) and dger on an n x n column-major f64 matrix, each
    launched warmup + steps times (for ncu captures on a bounded case)."""
    import torch

    from rblas_b200 import level2

    n = args.level2
    g = torch.Generator(device="cuda")
    g.manual_seed(9)
    A = torch.randn(n * n, dtype=torch.float64, device="cuda", generator=g)
    x = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
    y = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
    sh = torch.cuda.current_stream().cuda_stream
    out = {"level2": n}
    for name, fn, nbytes in (
            ("dgemv_N", lambda: level2.gemv_dev(1, 0, n, n, 1.0, A.data_ptr(), n, x.data_ptr(), 1, 0.5, y.data_ptr(),
                                                1, np.float64, stream=sh), 8.0 * n * n),
            ("dgemv_T", lambda: level2.gemv_dev(1, 1, n, n, 1.0, A.data_ptr(), n, x.data_ptr(), 1, 0.5, y.data_ptr(),
                                                1, np.float64, stream=sh), 8.0 * n * n),
            ("dger", lambda: level2.ger_dev(1, n, n, 1e-3, x.data_ptr(), 1, y.data_ptr(), 1, A.data_ptr(), n,
                                            np.float64, stream=sh), 16.0 * n * n)):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        for i in range(args.warmup + args.steps):
            if i == args.warmup:
                e0.record()
            fn()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / max(args.steps, 1)
        out[name] = {"ms": ms, "gb_s": nbytes / (ms * 1e-3) / 1e9}
    print(json.dumps(out))


def run_grouped_only(args):
    """The first `--grouped-batch N` requests of the serving stream as one
    grouped launch (device-resident operands), launched warmup + steps times
    (for ncu captures of the grouped kernel on a bounded batch)."""
    import torch

    from rblas_b200.serving import Problem, grouped_gemm

    tr = serving_trace(args.grouped_batch)
    g = torch.Generator(device="cuda")
    g.manual_seed(6)
    big = 4096 * 4096 + (1 << 22)
    pools = {0: torch.randn(big, dtype=torch.float32, device="cuda", generator=g),
             1: torch.randn(big, dtype=torch.float64, device="cuda", generator=g)}
    outs, probs, flops = [], [], 0.0
    for i in range(args.grouped_batch):
        m, n, k = (int(x) for x in tr["mnk"][i])
        dt = int(tr["dtype"][i])
        layout, ta, tb = int(tr["layout"][i]), int(tr["ta"][i]), int(tr["tb"][i])
        ar, ac = (k, m) if ta else (m, k)
        br, bc = (n, k) if tb else (k, n)
        lda = ar if layout == 1 else ac
        ldb = br if layout == 1 else bc
        ldc = m if layout == 1 else n
        es = 4 if dt == 0 else 8
        base = pools[dt].data_ptr()
        offs = [int(o) // 16 * 16 for o in tr["offs"][i]]
        c = torch.empty(m * n, dtype=torch.float32 if dt == 0 else torch.float64, device="cuda").normal_()
        outs.append(c)
        probs.append(Problem(np.float32 if dt == 0 else np.float64, layout, ta, tb, m, n, k, float(tr["alpha"][i]),
                             base + offs[0] * es, lda, base + offs[1] * es, ldb, float(tr["beta"][i]),
                             c.data_ptr(), ldc))
        flops += 2.0 * m * n * k
    sh = torch.cuda.current_stream().cuda_stream
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    for i in range(args.warmup + args.steps):
        if i == args.warmup:
            e0.record()
        grouped_gemm(probs, sh)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / max(args.steps, 1)
    print(json.dumps({"grouped_batch": args.grouped_batch, "flop": flops, "ms": ms,
                      "tflops": flops / (ms * 1e-3) / 1e12}))


def run_grouped_ozaki_only(args):
    """The f64 requests among the first `--grouped-ozaki N` requests of the
    serving stream in the Ozaki form (or, with `--grouped-bf16 N`, the f32
    ones in BF16X6): one grouped launch (rb_gemm_grouped_ozaki_dev /
    rb_gemm_grouped_bf16_dev) against one single-problem call per request in
    the same form and one grouped plain launch, warmup + steps times each."""
    import torch

    from rblas_b200 import level3
    from rblas_b200.serving import Problem, grouped_gemm, grouped_gemm_bf16, grouped_gemm_ozaki
    from rblas_b200.types import Precision

    f32 = args.grouped_bf16 > 0
    count = args.grouped_bf16 if f32 else args.grouped_ozaki
    npdt, tdt, es = (np.float32, torch.float32, 4) if f32 else (np.float64, torch.float64, 8)
    prec = Precision.Bf16x6 if f32 else Precision.Ozaki
    tr = serving_trace(count)
    g = torch.Generator(device="cuda")
    g.manual_seed(6)
    pool = torch.randn(4096 * 4096 + (1 << 22), dtype=tdt, device="cuda", generator=g)
    probs, flops = [], 0.0
    keep = []
    min_flop = args.min_flop
    for i in range(count):
        m, n, k = (int(x) for x in tr["mnk"][i])
        if int(tr["dtype"][i]) != (0 if f32 else 1) or 2.0 * m * n * k < min_flop:
            continue
        layout, ta, tb = int(tr["layout"][i]), int(tr["ta"][i]), int(tr["tb"][i])
        ar, ac = (k, m) if ta else (m, k)
        br, bc = (n, k) if tb else (k, n)
        lda = ar if layout == 1 else ac
        ldb = br if layout == 1 else bc
        ldc = m if layout == 1 else n
        offs = [int(o) // 16 * 16 for o in tr["offs"][i]]
        c = torch.empty(m * n, dtype=tdt, device="cuda").normal_()
        keep.append(c)
        probs.append(Problem(npdt, layout, ta, tb, m, n, k, float(tr["alpha"][i]),
                             pool.data_ptr() + offs[0] * es, lda, pool.data_ptr() + offs[1] * es, ldb,
                             float(tr["beta"][i]), c.data_ptr(), ldc))
        flops += 2.0 * m * n * k
    sh = torch.cuda.current_stream().cuda_stream

    def timed(fn):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        for i in range(args.warmup + args.steps):
            if i == args.warmup:
                e0.record()
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / max(args.steps, 1)

    def singles():
        for p in probs:
            level3.gemm_dev(p.layout, p.transa, p.transb, p.m, p.n, p.k, p.alpha, p.a, p.lda, p.b, p.ldb, p.beta,
                            p.c, p.ldc, npdt, prec=prec, stream=sh)

    form = "bf16x6" if f32 else "ozaki"
    grouped_form = (lambda: grouped_gemm_bf16(probs, prec, sh)) if f32 else (lambda: grouped_gemm_ozaki(probs, sh))
    out = {"requests": len(probs), "form": form, "min_flop": min_flop, "flop": flops}
    for name, fn in (("grouped_" + form, grouped_form), ("single_" + form, singles),
                     ("grouped_plain", lambda: grouped_gemm(probs, sh))):
        ms = timed(fn)
        out[name] = {"ms": ms, "tflops": flops / (ms * 1e-3) / 1e12}
    print(json.dumps(out))


def run_level3_only(args):
    """One complex GEMM (ConjTrans x NoTrans, `--cplx`) or one Level-3
    routine (`--level3 syrk|symm|trsm|trmm`, f64, n = k = the shape's N and K)
    on the `--kernel-only` shape, warmup + steps times (bounded ncu captures
    of the complex and Level-3 kernels)."""
    import torch

    from rblas_b200 import _lib, complex3
    from rblas_b200.types import Precision

    m, n, k = args.shape
    sh = torch.cuda.current_stream().cuda_stream
    g = torch.Generator(device="cuda")
    g.manual_seed(9)
    prec = {"plain": Precision.Plain, "ozaki": Precision.Ozaki, "bf16x3": Precision.Bf16x3,
            "bf16x6": Precision.Bf16x6}[args.form if args.form != "auto" else "plain"]
    dev_one = None  # the same routine on the device copies (trsm, trmm)
    if args.cplx:
        dt = torch.float64 if args.dtype == "f64" else torch.float32
        A, B, C = (torch.randn(2 * x, dtype=dt, device="cuda", generator=g) for x in (k * m, k * n, m * n))
        cdt = np.complex128 if args.dtype == "f64" else np.complex64

        def one():
            complex3.gemm_dev(2, 0, m, n, k, 1.0 + 0.5j, A.data_ptr(), k, B.data_ptr(), k, 0.0, C.data_ptr(), m, cdt,
                              prec=prec, stream=sh)
        work = 8.0 * m * n * k
    else:
        import ctypes as Cc
        lib = _lib.load()
        A = torch.randn(max(m, k) * max(m, k), dtype=torch.float64, device="cuda", generator=g) * 0.01
        A.view(max(m, k), max(m, k)).diagonal().uniform_(1.0, 2.0)
        B = torch.randn(max(m, k) * max(n, k), dtype=torch.float64, device="cuda", generator=g)
        C = torch.randn(m * max(n, m), dtype=torch.float64, device="cuda", generator=g)
        name = args.level3

        def pinned(t):
            h = torch.empty(t.numel(), dtype=t.dtype, pin_memory=True)
            h.copy_(t)
            return h.numpy()
        hA, hB, hC = (pinned(t) for t in (A, B, C))
        vp = lambda x: Cc.c_void_p(x.ctypes.data)  # noqa: E731
        err = _lib.RbError()
        if name == "syrk":
            def one():
                lib.rb_dsyrk(1, 0, m, k, 1.0, vp(hA), m, hA.size, 0.5, vp(hC), m, hC.size, Cc.byref(err))
            work = 1.0 * m * m * k
        elif name == "symm":
            def one():
                lib.rb_dsymm(0, 1, m, n, 1.0, vp(hA), m, hA.size, vp(hB), m, hB.size, 0.5, vp(hC), m, hC.size,
                             Cc.byref(err))
            work = 2.0 * m * m * n
        elif name == "trmm":
            def one():
                lib.rb_dtrmm(0, 1, 0, 0, m, n, 1.0, vp(hA), m, hA.size, vp(hB), m, hB.size, Cc.byref(err))

            def dev_one():
                lib.rb_dtrmm_dev(0, 1, 0, 0, m, n, 1.0, Cc.c_void_p(A.data_ptr()), m, Cc.c_void_p(B.data_ptr()),
                                 m, Cc.c_void_p(sh), Cc.byref(err))
            work = 1.0 * m * m * n
        else:
            def one():
                lib.rb_dtrsm(0, 1, 0, 0, m, n, 1.0, vp(hA), m, hA.size, vp(hB), m, hB.size, Cc.byref(err))

            def dev_one():
                lib.rb_dtrsm_dev(0, 1, 0, 0, m, n, 1.0, Cc.c_void_p(A.data_ptr()), m, Cc.c_void_p(B.data_ptr()),
                                 m, Cc.c_void_p(sh), Cc.byref(err))
            work = 1.0 * m * m * n
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    import time as _t

    def timed(fn):
        t0 = 0.0
        for i in range(args.warmup + args.steps):
            if i == args.warmup:
                torch.cuda.synchronize()
                e0.record()
                t0 = _t.perf_counter()
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / max(args.steps, 1), (_t.perf_counter() - t0) * 1e3 / max(args.steps, 1)
    ms, wall = timed(one)
    out = {"level3_only": args.level3 or "complex", "shape": [m, n, k], "ms": ms, "wall_ms": wall,
           "tflops": work / (ms * 1e-3) / 1e12}
    if dev_one is not None:
        dms, _ = timed(dev_one)
        out["device_ms"] = dms
        out["device_tflops"] = work / (dms * 1e-3) / 1e12
    print(json.dumps(out))


def run_trsm_batched_only(args):
    """The batched trsm of the C4 configuration (512 x 512 lower, 64
    right-hand sides; f64, or f32 with `--dtype f32`) on `--trsm-batched BATCH`
    members, launched warmup + steps times (for ncu captures on a bounded
    batch)."""
    import torch

    from rblas_b200 import level3

    q, nrhs, batch = 512, 64, args.trsm_batched
    tdt, ndt = (torch.float32, np.float32) if args.dtype == "f32" else (torch.float64, np.float64)
    g = torch.Generator(device="cuda")
    g.manual_seed(8)
    A = torch.randn(q * q * batch, dtype=tdt, device="cuda", generator=g) * (0.1 / q ** 0.5)
    A.view(batch, q, q).diagonal(dim1=1, dim2=2).uniform_(1.0, 2.0)
    B = torch.rand(q * nrhs * batch, dtype=tdt, device="cuda", generator=g) * 2 - 1
    sh = torch.cuda.current_stream().cuda_stream
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    for i in range(args.warmup + args.steps):
        if i == args.warmup:
            e0.record()
        level3.trsm_batched_dev(0, 1, 0, 0, q, nrhs, 1.0, A.data_ptr(), q, q * q, B.data_ptr(), q, q * nrhs,
                                batch, ndt, stream=sh)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / max(args.steps, 1)
    print(json.dumps({"trsm_batched": [q, nrhs, batch], "dtype": args.dtype, "ms": ms,
                      "tflops": q * q * nrhs * batch / (ms * 1e-3) / 1e12}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--form", choices=["auto", "plain", "ozaki", "bf16x3", "bf16x6"], default="auto")
    ap.add_argument("--no-sgemm", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--kernel-only", dest="shape", type=int, nargs=3, default=None,
                    metavar=("M", "N", "K"), help="time one column-major GEMM shape only")
    ap.add_argument("--dtype", choices=["f32", "f64"], default="f64")
    ap.add_argument("--level2", type=int, default=0, metavar="N",
                    help="time dgemv (N, T) and dger on an N x N f64 matrix only")
    ap.add_argument("--level1", type=int, default=0, metavar="N",
                    help="Level-1 calls on N-scalar f64 vectors only (bounded ncu captures)")
    ap.add_argument("--grouped-batch", type=int, default=0, metavar="N",
                    help="time one grouped launch of the first N serving requests only")
    ap.add_argument("--grouped-ozaki", type=int, default=0, metavar="N",
                    help="the f64 requests among the first N serving requests: grouped Ozaki vs single calls")
    ap.add_argument("--grouped-bf16", type=int, default=0, metavar="N",
                    help="the f32 requests among the first N serving requests: grouped BF16X6 vs single calls")
    ap.add_argument("--min-flop", type=float, default=1e9, help="--grouped-ozaki/-bf16: smallest request kept")
    ap.add_argument("--cplx", action="store_true", help="--kernel-only shape as a complex C/N GEMM")
    ap.add_argument("--level3", choices=["", "syrk", "symm", "trsm", "trmm"], default="",
                    help="--kernel-only shape through one f64 Level-3 host call")
    ap.add_argument("--trsm-batched", type=int, default=0, metavar="BATCH",
                    help="time the batched f64 trsm (512 x 512, 64 RHS) on BATCH members only")
    ap.add_argument("--serve", action="store_true", help="serving sweep (request stream replay)")
    ap.add_argument("--requests", type=int, default=20000)
    ap.add_argument("--rates", default="1000,2000,5000,8000,10000,12500,15000,17500,20000,25000,30000,35000,40000,50000")
    ap.add_argument("--no-autotune", action="store_true", help="serving: keep the built-in split-K rule")
    ap.add_argument("--serve-thresholds", default="", metavar="F32,F64",
                    help="serving: flop thresholds for the precision forms (default 2e8,1e9)")
    ap.add_argument("--no-serve", action="store_true", help="default run: skip the serving summary")
    ap.add_argument("--no-configs", action="store_true", help="default run: skip the C1/C3/C4 measurements")
    ap.add_argument("--budget-gb", type=float, default=120.0)
    ap.add_argument("--ta", type=int, default=0)
    ap.add_argument("--tb", type=int, default=0)
    args = ap.parse_args()
    if args.trsm_batched:
        run_trsm_batched_only(args)
    elif args.grouped_ozaki or args.grouped_bf16:
        run_grouped_ozaki_only(args)
    elif args.shape and (args.cplx or args.level3):
        run_level3_only(args)
    elif args.grouped_batch:
        run_grouped_only(args)
    elif args.level2:
        run_level2_only(args)
    elif args.level1:
        run_level1_only(args)
    elif args.serve:
        run_serve_mode(args)
    elif args.shape:
        run_kernel_only(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
