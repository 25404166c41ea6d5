"""The multi-GPU path of bench.py on the CPU: world_size 2 over gloo.

GEMM has no exchange step, so `bench.py --gpus N` runs one replica of the
step per rank; the ranks share only the barrier before each timed region and
the max over ranks of each time, and the whole-job value is every rank's work
over the slowest rank's time. These tests run that plumbing (bench.Replicas)
as two gloo ranks, and check that the reference arm does its work on rank 0
only.
"""
from __future__ import annotations

import json
import os
import socket
import subprocess
import sys

import pytest

torch = pytest.importorskip("torch")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    rep = bench.Replicas("gloo", torch.device("cpu"))
    rep.barrier()
    # each rank "timed" a different duration; the job's time is the slowest
    t = rep.max(1.0 + rank * 0.5)
    v = bench.Replicas.value(2.0e12, t, rep.ws)
    rep.close()
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump({"t": t, "value": v, "ws": rep.ws}, f)


def test_two_gloo_ranks_take_the_max_time_and_sum_the_work(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    res = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in range(2)]
    for r in res:
        assert r["ws"] == 2
        assert r["t"] == 1.5            # the slower rank's time on both ranks
        assert r["value"] == pytest.approx(2.0e12 * 2 / 1.5 / 1e12)


def test_single_process_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    env = {k: os.environ.get(k) for k in ("WORLD_SIZE", "RANK")}
    os.environ.pop("WORLD_SIZE", None)
    os.environ.pop("RANK", None)
    try:
        rep = bench.Replicas("gloo", torch.device("cpu"))
        assert rep.dist is None and rep.max(3.25) == 3.25
        rep.barrier()
        rep.close()
    finally:
        for k, v in env.items():
            if v is not None:
                os.environ[k] = v


def test_reference_arm_prints_on_rank_zero_only():
    """Under torchrun the other ranks of `--impl reference` exit 0 without work."""
    env = dict(os.environ, WORLD_SIZE="2", RANK="1", LOCAL_RANK="1")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                          "--steps", "1", "--warmup", "0"], capture_output=True, text=True, env=env, timeout=120)
    assert out.returncode == 0
    assert out.stdout.strip() == ""


def test_reference_arm_json_line():
    """`--impl reference` on one process prints one JSON line with the base
    contract's keys, the arm's CPU baseline and an e2e that moves no bytes
    (the restated CPU gemm runs on the host cores, no device involved)."""
    import json

    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "0"], capture_output=True, text=True, env=env, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config"):
        assert key in d, key
    assert d["value"] > 0 and d["higher_is_better"] is True and d["unit"] == "TFLOP/s"
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["sample"] and cb["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
