#!/usr/bin/env python
"""Benchmark: matrix-free H*psi on the periodic XXZ chain L=28, Delta=1.0,
sector N=14, k=0 (TranslationalBasis, D = 1,432,860 representatives, FP64).

A step is one H*psi over the whole sector vector.  `value` is the matvec's
algorithmic HBM bandwidth (GB/s) with the inputs resident in HBM and L2
flushed between steps; `e2e` is the same metric through the C ABI with host
buffers (host->device copy of psi and device->host copy of H*psi inside the
timed region).  Time-to-E0 (FP64 vs mixed precision Lanczos) is reported
beside it.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

For N > 1 the driver launches one process per GPU (torchrun); every rank runs
an independent replica of the sector (the single-sector matvec has no
exchange step), `value` aggregates all ranks over the max-over-ranks time.
`--impl reference` times the CPU restatement of EDKit's threaded `mul`
(column scatter, thread-private outputs) on this host's cores.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

L, N, K_MOM, DELTA = 28, 14, 0, 1.0
METRIC = "matvec HBM GB/s"
WORKLOAD = "periodic XXZ chain L=28 Delta=1.0, TranslationalBasis N=14 k=0 (D=1432860), FP64 H*psi"
FALLBACK_HBM_GBS = 6650.0
L2_FLUSH_BYTES = 256 << 20


def algorithmic_bytes(states: np.ndarray, L: int, s_state=8, s_R=8, s_y=8, s_x=8, nvec=1):
    """D*(s_state + s_R + nvec*s_y) + nnz*nvec*s_x, nnz = every (row, col) hit
    including the merged diagonal: 1 + #antiparallel bonds of the ring per row."""
    s = states.astype(np.uint64)
    mask = np.uint64((1 << L) - 1)
    rot = ((s << np.uint64(1)) | (s >> np.uint64(L - 1))) & mask
    x = s ^ rot
    cnt = np.zeros(len(s), dtype=np.int64)
    while np.any(x):
        cnt += (x & np.uint64(1)).astype(np.int64)
        x >>= np.uint64(1)
    nnz = int(len(s) + cnt.sum())
    D = len(s)
    return D * (s_state + s_R + nvec * s_y) + nnz * nvec * s_x, nnz


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def profiled_traffic():
    """dram bytes per launch of the matvec kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "k_apply_trans0_L28_f64.md")
    if not os.path.exists(p):
        return None
    m = re.search(r"dram_bytes_per_launch:\s*([0-9.eE+]+)", open(p).read())
    return float(m.group(1)) if m else None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 6:
                continue
            try:
                sm.append(float(parts[0]))
                mx = max(mx, float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[2:]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def build_problem(ek):
    b = ek.TranslationalBasis(L=L, N=N, k=K_MOM)
    H = ek.trans_inv_operator(ek.spin((1.0, "xx"), (1.0, "yy"), (DELTA, "zz")), 2, b)
    return b, H


def run_gpu(args):
    import torch
    import torch.distributed as dist
    import __graft_entry__ as ge
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    ek = ge.load_package()
    from edkit_b200 import _lib as E
    lib = E.load()
    b, H = build_problem(ek)
    D = b.size(1)
    balg, nnz = algorithmic_bytes(b.I - 1, L)
    dev = torch.device("cuda", local)
    g = torch.Generator(device="cpu").manual_seed(1234)
    x = torch.randn(D, dtype=torch.float64, generator=g).to(dev)
    y = torch.empty(D, dtype=torch.float64, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def matvec():
        E.check(lib.edk_apply_async(H._h, E.F64, x.data_ptr(), y.data_ptr(), 1, D, D, 0,
                                    stream.cuda_stream))

    for _ in range(args.warmup):
        flush.fill_(1.0)
        matvec()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        t0 = time.perf_counter()
        for i in range(args.steps):
            flush.fill_(float(i))          # evict L2 between steps (outside the events)
            ev[i][0].record(stream)
            matvec()
            ev[i][1].record(stream)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
    if world > 1:
        dist.barrier()
    ms = [a.elapsed_time(c) for a, c in ev]
    ms_mean = float(np.mean(ms))
    t_max = torch.tensor([ms_mean], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t_max, op=dist.ReduceOp.MAX)
    ms_step = float(t_max.item())
    value = balg * world / (ms_step * 1e-3) / 1e9
    achieved = balg / (ms_mean * 1e-3) / 1e9

    # end to end through the C ABI with pinned host buffers
    xh = torch.randn(D, dtype=torch.float64, generator=g).pin_memory()
    yh = torch.empty(D, dtype=torch.float64).pin_memory()
    n_e2e = max(3, min(args.steps, 50))
    for _ in range(3):
        E.check(lib.edk_apply(H._h, E.F64, xh.data_ptr(), yh.data_ptr(), 1, D, D, 0, E.HOST))
    if world > 1:
        dist.barrier()
    te = []
    for _ in range(n_e2e):
        t1 = time.perf_counter()
        E.check(lib.edk_apply(H._h, E.F64, xh.data_ptr(), yh.data_ptr(), 1, D, D, 0, E.HOST))
        te.append(time.perf_counter() - t1)
    e2e_t = torch.tensor([float(np.mean(te))], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    e2e_val = balg * world / e2e_t.item() / 1e9

    # correctness guard on the benchmarked product (rank-local)
    ref = (H * x.cpu().numpy())
    err = float(np.linalg.norm(y.cpu().numpy() - ref) / np.linalg.norm(ref))

    result = None
    if rank == 0:
        peak, src = measured_peak()
        traffic = profiled_traffic()
        result = {
            "metric": METRIC, "value": round(value, 2), "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 5),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded normal psi)",
            "config": {"workload": WORKLOAD, "D": D, "nnz_hits": nnz,
                       "algorithmic_bytes_per_step": balg,
                       "parallelism": f"replicas{world}",
                       "l2": "flushed between steps (256 MiB write)",
                       "wall_s_timed_region": round(wall, 4)},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 4),
                         "traffic": traffic, "peak_source": src},
            "e2e": {"value": round(e2e_val, 3), "unit": "GB/s", "h2d_bytes_per_step": D * 8,
                    "d2h_bytes_per_step": D * 8, "ms_per_step": round(e2e_t.item() * 1e3, 4)},
            "gpu_launches": args.steps,
            "clocks": clk.summary(),
            "check_rel_err_vs_second_run": err,
        }
        if not args.skip_e0:
            result["time_to_e0"] = time_to_e0(ek, H, D)
        if world == 1 and not args.skip_cpu:
            result["cpu_baseline"] = cpu_baseline(balg, D, budget_s=args.cpu_budget)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if result is not None:
        print(json.dumps(result), flush=True)


def time_to_e0(ek, H, D):
    """FP64 vs mixed-precision Lanczos to a converged E0 (same start vector).
    Each variant runs twice; the second call is reported (workspace pool warm)."""
    v0 = np.random.default_rng(1234).standard_normal(D)
    out = {}
    for _ in range(2):
        e64, d64 = ek.lanczos_e0(H, v0, m=300, tol=1e-12, check_every=10)
    for _ in range(2):
        emx, dmx = ek.lanczos_e0(H, v0, m=300, tol=1e-12, check_every=10, precision="mixed",
                                 refine_steps=20)

    def phases(d):
        return {k: round(d[k], 5) for k in ("seconds_setup", "seconds_stage1", "seconds_refine")}

    out["fp64"] = {"seconds": round(d64["seconds"], 4), "E0": e64[0], "steps": d64["steps"],
                   "checks": d64["checks"], **phases(d64)}
    out["mixed"] = {"seconds": round(dmx["seconds"], 4), "E0": emx[0],
                    "steps_fp32": dmx["steps_low"], "steps_fp64_refine": dmx["steps"],
                    "refine_rounds": dmx["refine_rounds"], "checks": dmx["checks"], **phases(dmx)}
    out["dE0_rel_mixed_vs_fp64"] = abs(emx[0] - e64[0]) / abs(e64[0])
    out["speedup_mixed_vs_fp64"] = round(d64["seconds"] / dmx["seconds"], 3)
    return out


def cpu_sample(balg, D, budget_s, nthreads=0):
    """Time the CPU restatement of EDKit's threaded mul on a column sample."""
    import oracle as O
    o = O.translational(L, k=K_MOM, N=N)
    Ho = O.trans_inv_operator(O.spin((1.0, "xx"), (1.0, "yy"), (DELTA, "zz")), 2, o)
    x = np.random.default_rng(1234).standard_normal(D)
    cal = max(256, D // 256)
    t = time.perf_counter()
    Ho.mul_cols(x, 1, cal, nthreads)
    t_cal = time.perf_counter() - t
    return O, Ho, x, t_cal / cal


def cpu_baseline(balg, D, budget_s=15.0):
    O, Ho, x, per_col = cpu_sample(balg, D, budget_s)
    cols = int(min(D, max(1024, budget_s / max(per_col, 1e-9))))
    t = time.perf_counter()
    Ho.mul_cols(x, 1, cols)
    dt = time.perf_counter() - t
    cores = O.lib().orc_num_threads()
    return {"value": round(balg * cols / D / dt / 1e9, 6), "unit": "GB/s", "cores": cores,
            "kind": "port",
            "sample": f"{cols} of {D} input columns of one H*psi (EDKit mul: column scatter, "
                      f"thread-private outputs), {dt:.2f} s"}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import oracle as O
    o = O.translational(L, k=K_MOM, N=N)
    Ho = O.trans_inv_operator(O.spin((1.0, "xx"), (1.0, "yy"), (DELTA, "zz")), 2, o)
    I, _ = o.tables()
    D = len(I)
    balg, nnz = algorithmic_bytes(I - 1, L)
    x = np.random.default_rng(1234).standard_normal(D)
    cal = max(256, D // 256)
    t = time.perf_counter()
    Ho.mul_cols(x, 1, cal)
    per_col = (time.perf_counter() - t) / cal
    total_budget = args.ref_budget
    cols = int(min(D, max(256, total_budget / max(args.steps + args.warmup, 1) /
                       max(per_col, 1e-9))))
    for i in range(args.warmup):
        Ho.mul_cols(x, 1 + (i * cols) % (D - cols + 1), (i * cols) % (D - cols + 1) + cols)
    ts = []
    for i in range(args.steps):
        j0 = 1 + (i * cols) % (D - cols + 1)
        t = time.perf_counter()
        Ho.mul_cols(x, j0, j0 + cols - 1)
        ts.append(time.perf_counter() - t)
    ms = float(np.mean(ts)) * 1e3
    value = balg * cols / D / (ms * 1e-3) / 1e9
    cores = O.lib().orc_num_threads()
    sample = (f"{cols} of {D} input columns per step of one H*psi (C++ restatement of "
              f"EDKit mul: column scatter, thread-private outputs; Julia is not installed)")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(value, 6), "unit": "GB/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded normal psi)",
        "config": {"workload": WORKLOAD, "D": D, "nnz_hits": nnz,
                   "algorithmic_bytes_per_step": balg * cols // D,
                   "parallelism": f"host threads x{cores}"},
        "cpu_baseline": {"value": round(value, 6), "unit": "GB/s", "cores": cores,
                         "kind": "port", "sample": sample},
        "e2e": {"value": round(value, 6), "unit": "GB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--skip-e0", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--ref-budget", type=float, default=120.0)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
