"""RFP Cholesky+solve benchmark (one JSON line on rank 0).

Workload: n = 32768, transr='T', uplo='U', C = A A^T + 1.0 I with
A ~ N(0,1)/sqrt(k), k = 1024 (synthetic, seeded, built on the device by the
library's own ssfrk), 64 right-hand sides B ~ N(0,1).
One step = spftrf (in-place Cholesky) + spftrs (64 RHS) on a fresh copy of C.
Metric: Cholesky+solve TFLOP/s = (n^3/3 + 2 n^2 nrhs) / time.
The RFP matrix (2.1 GB) is larger than L2 (126 MB), so no extra L2 flush.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--math fp32|bf16x3] [--n 32768] [--nrhs 64]

--impl reference times the reference's algorithm on the host cores: LAPACK's
RFP routines (ssfrk/spftrf/spftrs via scipy/OpenBLAS, all threads), which the
reference's GPU code translates call for call; each step is a bounded sample
(n = 8192) of the same workload.  N > 1 GPUs run independent replicas
(the path has no cross-GPU exchange); value = total flops / max-rank time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "RFP Cholesky+solve TFLOP/s at n=32768 (spftrf + spftrs 64 RHS)"


def chol_solve_flops(n: int, nrhs: int) -> float:
    return n ** 3 / 3.0 + n ** 2 / 2.0 + n / 6.0 + 2.0 * n * n * nrhs


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows: list[list[str]] = []
        self._stop = threading.Event()
        self._proc = None

    def __enter__(self):
        try:
            self._proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self._proc = None
        return self

    def _read(self):
        for line in self._proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *exc):
        if self._proc is not None:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except Exception:
                self._proc.kill()

    def summary(self) -> dict:
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows if len(r) > 8
                          for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def dist_setup():
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(local)
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cpu_baseline(n_sample: int = 8192, nrhs: int = 64, reps: int = 2) -> dict:
    """LAPACK (scipy/OpenBLAS) on the host: spftrf + spftrs at n_sample."""
    import numpy as np

    from oracle import port
    rng = np.random.default_rng(0)
    k = n_sample // 32
    A = (rng.standard_normal((n_sample, k)) / np.sqrt(k)).astype(np.float32)
    B = rng.standard_normal((n_sample, nrhs)).astype(np.float32)
    best = None
    for _ in range(reps):
        r = port.cholesky_solve(A, B, 1.0)
        t = r["spftrf"] + r["spftrs"]
        best = t if best is None else min(best, t)
    val = chol_solve_flops(n_sample, nrhs) / best / 1e12
    return {"value": round(val, 4), "unit": "TFLOP/s", "cores": port.threads(),
            "kind": "port",
            "sample": f"LAPACK spftrf+spftrs (scipy/OpenBLAS) at n={n_sample}, k={k}, "
                      f"nrhs={nrhs}, transr=T uplo=U, best of {reps}"}


def run_reference(args, rank, world):
    if rank != 0:
        return
    for _ in range(max(0, args.warmup)):
        cpu_baseline(reps=1)
    vals = [cpu_baseline(reps=1)["value"] for _ in range(args.steps)]
    cb = cpu_baseline(reps=1)
    v = statistics.median(vals)
    n_s = 8192
    ms = chol_solve_flops(n_s, args.nrhs) / (v * 1e12) * 1e3
    cb["value"] = v
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "TFLOP/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"RFP Cholesky+solve, host LAPACK sample n={n_s}, "
                                   f"nrhs={args.nrhs}, transr=T, uplo=U",
                       "n": n_s, "nrhs": args.nrhs, "parallelism": "replicas"},
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "TFLOP/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args, rank, world, local):
    import torch

    import curfp_b200 as curfp
    from curfp_b200 import _lib

    n, k, nrhs = args.n, args.k, args.nrhs
    flops = chol_solve_flops(n, nrhs)
    nt = n * (n + 1) // 2
    dev = torch.device("cuda", local)
    g = torch.Generator(device=dev).manual_seed(1234 + rank)
    A = torch.randn(n, k, device=dev, generator=g) / k ** 0.5
    B0 = torch.randn(n, nrhs, device=dev, generator=g)
    C0 = torch.empty(nt, device=dev)
    curfp.ssfrk(A, C0)
    curfp.add_to_diagonal(C0, 1.0)
    del A
    C = torch.empty_like(C0)
    Bc = B0.t().contiguous()         # column-major n x nrhs for the C ABI
    X = torch.empty_like(Bc)
    h = curfp._get_handle()
    lib = _lib.load()
    import ctypes
    info = ctypes.c_int(0)

    def step():
        st = lib.curfpSpftrf(h.ptr, 1, 1, n, ctypes.c_void_p(C.data_ptr()), ctypes.byref(info))
        assert st == 0 and info.value == 0, (st, info.value)
        st = lib.curfpSpftrs(h.ptr, 1, 1, n, nrhs, ctypes.c_void_p(C.data_ptr()),
                             ctypes.c_void_p(X.data_ptr()), n)
        assert st == 0

    for _ in range(args.warmup):
        C.copy_(C0)
        X.copy_(Bc)
        step()
    torch.cuda.synchronize()

    times = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            C.copy_(C0)
            X.copy_(Bc)
            barrier(world)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            step()
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
    total_ms = max_over_ranks(sum(times), world)
    ms_step = total_ms / args.steps
    value = world * args.steps * flops / (total_ms * 1e-3) / 1e12

    # End to end through the C ABI with host buffers: H2D of the RFP matrix
    # and B (pinned), factor + solve, D2H of X.
    e2e = None
    if not args.no_e2e:
        C_h = C0.cpu().pin_memory()
        B_h = Bc.cpu().pin_memory()
        X_h = torch.empty_like(B_h).pin_memory()
        e2e_times = []
        for i in range(args.warmup + args.steps):
            barrier(world)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            C.copy_(C_h, non_blocking=True)
            X.copy_(B_h, non_blocking=True)
            step()
            X_h.copy_(X, non_blocking=True)
            e1.record()
            torch.cuda.synchronize()
            if i >= args.warmup:
                e2e_times.append(e0.elapsed_time(e1))
        e2e_ms = max_over_ranks(sum(e2e_times), world)
        e2e = {"value": round(world * args.steps * flops / (e2e_ms * 1e-3) / 1e12, 4),
               "unit": "TFLOP/s", "h2d_bytes_per_step": nt * 4 + n * nrhs * 4,
               "d2h_bytes_per_step": n * nrhs * 4 + 4}

    cb = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cb = cpu_baseline()

    if rank == 0:
        line = {"metric": METRIC, "value": round(value, 4), "unit": "TFLOP/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": round(ms_step, 3), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic",
                "config": {"workload": f"RFP Cholesky+solve n={n} k={k} nrhs={nrhs} "
                                       f"transr=T uplo=U shift=1.0 math={args.math}",
                           "n": n, "k": k, "nrhs": nrhs, "math": args.math,
                           "parallelism": f"replicas{world}",
                           "l2": "inputs (2.1 GB RFP) larger than L2, no flush"},
                "clocks": clk.summary(), "e2e": e2e, "cpu_baseline": cb}
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--math", default="fp32", choices=["fp32", "bf16x3"])
    ap.add_argument("--n", type=int, default=32768)
    ap.add_argument("--k", type=int, default=1024)
    ap.add_argument("--nrhs", type=int, default=64)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        run_reference(args, rank, world)
        return
    rank, world, local = dist_setup()
    try:
        run_ours(args, rank, world, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
