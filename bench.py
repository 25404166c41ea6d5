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


def dist_info():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


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

def run_ours(args):
    import torch

    import rblas_b200 as rb
    from rblas_b200 import _lib, level3
    from rblas_b200.types import Layout, Precision

    ws, rank, local = dist_info()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))

    rb.load_library()
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

    def timed(prec, steps, warmup):
        for _ in range(warmup):
            dev_step(prec)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        l0 = rb.launch_count()
        e0.record(stream)
        for _ in range(steps):
            dev_step(prec)
        e1.record(stream)
        torch.cuda.synchronize()
        launches = rb.launch_count() - l0
        ms = e0.elapsed_time(e1)
        if dist:
            t = torch.tensor([ms], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms / steps, launches

    forms = {}
    headline = Precision.Plain
    candidates = [("plain", Precision.Plain)]
    if args.form in ("auto", "ozaki"):
        candidates.append(("ozaki", Precision.Ozaki))
    clocks = None
    for name, prec in candidates:
        try:
            dev_step(prec)
            torch.cuda.synchronize()
        except rb.BlasError as e:
            forms[name] = {"unavailable": str(e)}
            continue
        with ClockSampler(local) as cs:
            ms, launches = timed(prec, args.steps, args.warmup)
        forms[name] = {"tflops": step_flops() * ws / (ms * 1e-3) / 1e12, "ms_per_step": ms,
                       "gpu_launches": launches}
        csum = cs.summary()
        forms[name]["clocks"] = csum
        if name == "ozaki" or headline == Precision.Plain:
            headline_name = name
            headline = prec
            clocks = csum
    if args.form == "plain":
        headline_name = "plain"
    hl = forms[headline_name]
    err_status = rb.device_error()

    # ---- roofline of the dominant kernel: time one 4096^3 N/N launch alone
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    reps = 3
    e0.record(stream)
    for _ in range(reps):
        level3.gemm_dev(Layout.RowMajor, 0, 0, BIG, BIG, BIG, ALPHA, A.data_ptr(), BIG, B.data_ptr(),
                        BIG, BETA, Cs[0].data_ptr(), BIG, np.float64, prec=headline, stream=sh)
    e1.record(stream)
    torch.cuda.synchronize()
    kernel_ms = e0.elapsed_time(e1) / reps
    f64_peak = float(_lib.load().rb_probe_fma_peak_tflops(1, 0))
    achieved = 2.0 * BIG ** 3 / (kernel_ms * 1e-3) / 1e12
    roofline = {"bound": "fp64" if headline == Precision.Plain else "tensor",
                "achieved": achieved, "peak": f64_peak, "unit": "TFLOP/s",
                "frac": achieved / f64_peak if f64_peak > 0 else None, "traffic": None,
                "kernel": "simt_gemm_kernel<double> (one 4096^3 launch)",
                "peak_source": "FP64 DFMA throughput measured in-run by rb_probe_fma_peak_tflops "
                               "(not in MEASURED_PEAKS.json)"}

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
        na = {id(t): t.numpy() for t in [hA, hB, hA2, hB2, hC2] + hC}

        def host_step(prec):
            h2d = d2h = 0
            for i, (ta, tb, m, n, k) in enumerate(step_gemms()):
                if m == BIG:
                    a, b, c = na[id(hA)], na[id(hB)], na[id(hC[i])]
                else:
                    a, b, c = na[id(hA2)], na[id(hB2)], na[id(hC2)]
                level3.gemm(Layout.RowMajor, ta, tb, m, n, k, ALPHA, a, m if ta else k, b,
                            k if tb else n, BETA, c, n, prec=prec)
                h2d += (a.nbytes + b.nbytes + c.nbytes)
                d2h += c.nbytes
            return h2d, d2h

        for _ in range(max(1, args.warmup)):
            host_step(headline)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        k_e2e = max(2, args.steps // 2)
        t0 = time.perf_counter()
        for _ in range(k_e2e):
            h2d, d2h = host_step(headline)
        torch.cuda.synchronize()
        dt = (time.perf_counter() - t0) / k_e2e
        if dist:
            t = torch.tensor([dt], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            dt = float(t.item())
        e2e = {"value": step_flops() * ws / dt / 1e12, "unit": "TFLOP/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "steps": k_e2e,
               "timing": "host wall clock around synchronous API calls"}

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
            "roofline": roofline, "cpu_baseline": cpu,
            "device_error": err_status[0],
        }
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


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
    prec = {"plain": Precision.Plain, "ozaki": Precision.Ozaki, "bf16x3": Precision.Bf16x3}[
        args.form if args.form != "auto" else "plain"]
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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--form", choices=["auto", "plain", "ozaki"], default="auto")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--kernel-only", dest="shape", type=int, nargs=3, default=None,
                    metavar=("M", "N", "K"), help="time one column-major GEMM shape only")
    ap.add_argument("--dtype", choices=["f32", "f64"], default="f64")
    ap.add_argument("--ta", type=int, default=0)
    ap.add_argument("--tb", type=int, default=0)
    args = ap.parse_args()
    if args.shape:
        run_kernel_only(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
