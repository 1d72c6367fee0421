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
The natural shard of the batched workloads, the 512-instance disorder
ensemble split over the ranks (strong scaling), is reported beside it as
`ensemble_sharded` at every N.
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


def profiled_traffic(search="rank"):
    """dram bytes per launch of the matvec kernel from the committed ncu summary."""
    name = "k_apply_plan_rank_L28_f64.md" if search == "rank" else "k_apply_trans0_L28_f64.md"
    p = os.path.join(ROOT, "profiles", name)
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
                 "--format=csv,noheader,nounits", "-lms", "50"],
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


def build_problem(ek, search="rank"):
    b = ek.TranslationalBasis(L=L, N=N, k=K_MOM)
    H = ek.trans_inv_operator(ek.spin((1.0, "xx"), (1.0, "yy"), (DELTA, "zz")), 2, b)
    b.set_search(search)  # index search of the target rows (the autotuner's pick here: rank)
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
    b, H = build_problem(ek, args.search)
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
    with ClockSampler(local) as clk:
        # the same steps, untimed, for about a second before the timed region:
        # the clock samples cover this soak and the timed steps that follow it
        t_soak = time.perf_counter()
        while time.perf_counter() - t_soak < args.clock_soak:
            for _ in range(50):
                flush.fill_(1.0)
                matvec()
            torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
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

    # the same kernel with the hash-table search, for comparison
    other = None
    if args.search != "hash":
        b.set_search("hash")
        for _ in range(3):
            flush.fill_(1.0)
            matvec()
        torch.cuda.synchronize()
        n_o = min(args.steps, 200)
        evo = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(n_o)]
        for i in range(n_o):
            flush.fill_(float(i))
            evo[i][0].record(stream)
            matvec()
            evo[i][1].record(stream)
        torch.cuda.synchronize()
        ms_h = float(np.mean([a.elapsed_time(c) for a, c in evo]))
        other = {"search": "hash", "ms_per_step": round(ms_h, 5),
                 "GB_s_algorithmic": round(balg / (ms_h * 1e-3) / 1e9, 2),
                 "speedup_of_headline_search": round(ms_h / ms_mean, 3)}
        b.set_search(args.search)

    # the same product from the cached matrix (sparse!(opt) on the device)
    mat = None
    if not args.skip_materialized:
        y_free = H * x.cpu().numpy()
        entries = H.sparse_()
        for _ in range(args.warmup):
            flush.fill_(1.0)
            matvec()
        torch.cuda.synchronize()
        evm = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(args.steps)]
        for i in range(args.steps):
            flush.fill_(float(i))
            evm[i][0].record(stream)
            matvec()
            evm[i][1].record(stream)
        torch.cuda.synchronize()
        ms_m = float(np.mean([a.elapsed_time(c) for a, c in evm]))
        ref_m = y_free
        mat = {"ms_per_step": round(ms_m, 5), "GB_s_algorithmic": round(balg / ms_m / 1e6, 2),
               "entries": entries,
               "frac_of_measured_hbm": round(balg / ms_m / 1e6 / measured_peak()[0], 4),
               "rel_diff_vs_matrix_free": float(
                   np.linalg.norm(ref_m - y.cpu().numpy()) / np.linalg.norm(ref_m))}
        H.clear_sparse_cache_()

    # a block of 64 right-hand sides: one SpMM (each hit located once for all
    # columns) against 64 single-vector passes, matrix-free and materialised
    blk = None
    if not args.skip_materialized:
        nb = 64
        X = torch.randn((nb, D), dtype=torch.float64, generator=g).to(dev)
        Y = torch.empty_like(X)

        def blockmv():
            E.check(lib.edk_apply_async(H._h, E.F64, X.data_ptr(), Y.data_ptr(), nb, D, D, 0,
                                        stream.cuda_stream))

        def timed(reps=5):
            for _ in range(2):
                flush.fill_(1.0)
                blockmv()
            torch.cuda.synchronize()
            evb = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                   for _ in range(reps)]
            for i in range(reps):
                flush.fill_(float(i))
                evb[i][0].record(stream)
                blockmv()
                evb[i][1].record(stream)
            torch.cuda.synchronize()
            return float(np.median([a.elapsed_time(c) for a, c in evb]))

        blk = {"nvec": nb}
        bb = D * (8 + 8 + nb * 8) + nnz * nb * 8
        for name, mat_on in (("matrix_free", False), ("materialized", True)):
            if mat_on:
                H.sparse_()
            H.configure_("fast", 1, block=False)
            t_cols = timed()
            Yc = Y.clone()
            H.configure_("fast", 1, block=True)
            t_blk = timed()
            blk[name] = {"ms_spmm": round(t_blk, 4), "ms_one_column_at_a_time": round(t_cols, 4),
                         "speedup": round(t_cols / t_blk, 2),
                         "GB_s_algorithmic_spmm": round(bb / t_blk / 1e6, 1),
                         "rel_diff": float((torch.linalg.norm(Y - Yc) / torch.linalg.norm(Yc)).item())}
        H.clear_sparse_cache_()
        del X, Y, Yc

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

    # the natural shard of the batched workloads: the disorder ensemble over the ranks
    shard = ensemble_sharded(ek, rank, world, dev) if not args.skip_e0 else None

    # correctness guard on the benchmarked product (rank-local)
    ref = (H * x.cpu().numpy())
    err = float(np.linalg.norm(y.cpu().numpy() - ref) / np.linalg.norm(ref))

    result = None
    if rank == 0:
        peak, src = measured_peak()
        traffic = profiled_traffic(args.search)
        result = {
            "metric": METRIC, "value": round(value, 2), "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 5),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded normal psi)",
            "config": {"workload": WORKLOAD, "D": D, "nnz_hits": nnz,
                       "algorithmic_bytes_per_step": balg,
                       "index_search": args.search,
                       "parallelism": f"replicas{world}",
                       "l2": "flushed between steps (256 MiB write)",
                       "wall_s_timed_region": round(wall, 4),
                       "clock_window": f"nvidia-smi every 50 ms over a {args.clock_soak:g} s "
                                       "soak of the same steps and the timed steps after it"},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 4),
                         "traffic": traffic, "peak_source": src},
            "e2e": {"value": round(e2e_val, 3), "unit": "GB/s", "h2d_bytes_per_step": D * 8,
                    "d2h_bytes_per_step": D * 8, "ms_per_step": round(e2e_t.item() * 1e3, 4)},
            "gpu_launches": args.steps,
            "clocks": clk.summary(),
            "check_rel_err_vs_second_run": err,
        }
        if other is not None:
            result["matvec_other_search"] = other
        if mat is not None:
            result["matvec_materialized"] = mat
        if blk is not None:
            result["block_rhs_64"] = blk
        if shard is not None:
            result["ensemble_sharded"] = shard
        if not args.skip_e0:
            result["time_to_e0"] = time_to_e0(ek, H, D)
            # the batched workloads: every momentum sector of one chain, and a
            # disorder ensemble, FP64 against mixed precision
            result["config4_momentum_sectors"] = config4_sectors(ek, block=args.extras)
            result["config5_random_field_ensemble"] = config5_ensemble(ek)
        if args.extras:
            result["config1_tensor_L16"] = config1_tensor(ek)
            result["config3_krylov_L32"] = config3_krylov(ek)
        if world == 1 and not args.skip_cpu:
            result["cpu_baseline"] = cpu_baseline(balg, D, budget_s=args.cpu_budget)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if result is not None:
        print(json.dumps(result), flush=True)


def ensemble_sharded(ek, rank, world, dev):
    """The 512-instance random-field ensemble (the config-5 instances) split
    over the ranks by edkit_b200.sharding (longest-processing-time packing of
    D * L per instance): each rank builds and solves only its share (mixed
    precision batched Lanczos for E0, tol 1e-12), the eigenvalues are gathered
    at the end, no collective on the data path.  Strong scaling over the fixed
    ensemble: the time is the solve's, max over ranks (CUDA events around the
    synchronous call on each rank, then an all-reduce MAX)."""
    import torch
    import torch.distributed as dist
    from math import comb
    from edkit_b200.sharding import partition
    rng = np.random.default_rng(2024)
    specs = []
    for _ in range(512):
        Lq = int(rng.choice([12, 14, 16, 18, 20]))
        specs.append((Lq, rng.uniform(-3, 3, Lq)))
    w = [comb(Lq, Lq // 2) * Lq for Lq, _ in specs]
    mine = partition(w, world)[rank]
    bond = ek.spin((1.0, "xx"), (1.0, "yy"), (1.0, "zz"))
    ops, v0s = [], []
    for qi in mine:
        Lq, h = specs[qi]
        mats = [bond] * (Lq - 1) + [hi * ek.spin("z") for hi in h]
        inds = [[i, i + 1] for i in range(1, Lq)] + [[i] for i in range(1, Lq + 1)]
        ops.append(ek.operator(mats, inds, ek.ProjectedBasis(L=Lq, N=Lq // 2)))
        v0s.append(np.random.default_rng(qi).standard_normal(ops[-1].size(1)))
    ek.batch_lanczos_e0(ops, v0s, m=200, nev=1, tol=1e-12, check_every=10, precision="mixed")
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    a, c = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    ev, d = ek.batch_lanczos_e0(ops, v0s, m=200, nev=1, tol=1e-12, check_every=10,
                                precision="mixed")
    c.record()
    torch.cuda.synchronize()
    t = torch.tensor([a.elapsed_time(c) * 1e-3], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        got = [None] * world
        dist.all_gather_object(got, (mine, ev[:, 0].tolist()))
        e0 = np.full(len(specs), np.nan)
        for idx, vals in got:
            e0[idx] = vals
    else:
        e0 = ev[:, 0]
    return {"instances": len(specs), "ranks": world, "rows_this_rank": int(sum(op.size(1) for op in ops)),
            "instances_this_rank": len(mine), "seconds_max_over_ranks": round(float(t.item()), 4),
            "scaling": "strong", "all_gathered": bool(np.all(np.isfinite(e0))),
            "E0_sum": float(np.sum(e0))}


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
    # same two runs on the cached matrix (sparse!(opt)); the build is timed too
    t = time.perf_counter()
    H.sparse_()
    build = time.perf_counter() - t
    for _ in range(2):
        e64m, d64m = ek.lanczos_e0(H, v0, m=300, tol=1e-12, check_every=10)
    for _ in range(2):
        emxm, dmxm = ek.lanczos_e0(H, v0, m=300, tol=1e-12, check_every=10, precision="mixed",
                                   refine_steps=20)
    H.clear_sparse_cache_()
    out["materialized"] = {
        "build_seconds": round(build, 4),
        "fp64_seconds": round(d64m["seconds"], 4), "mixed_seconds": round(dmxm["seconds"], 4),
        "fp64_steps": d64m["steps"], "mixed_steps_fp32": dmxm["steps_low"],
        "speedup_mixed_vs_fp64": round(d64m["seconds"] / dmxm["seconds"], 3),
        "speedup_mixed_materialized_vs_fp64_matrix_free": round(d64["seconds"] / dmxm["seconds"], 3),
        "dE0_rel_mixed_vs_fp64": abs(emxm[0] - e64[0]) / abs(e64[0])}
    return out


def config1_tensor(ek, steps=150):
    """Open XXZ L=16, Delta=1.5 on the TensorBasis (D=65536), ComplexF64 psi
    with seeded normal parts, normalised: one H*psi and a 150-step Lanczos for
    E0 on the GPU; the oracle's threaded mul on the host for the same psi."""
    import torch
    import oracle as O
    L = 16
    b = ek.TensorBasis(L=L)
    inds = [[i, i + 1] for i in range(1, L)]
    bond = ek.spin((1.0, "xx"), (1.0, "yy"), (1.5, "zz"))
    H = ek.operator([bond] * (L - 1), inds, b)
    rng = np.random.default_rng(1234)
    psi = rng.standard_normal(2 ** L) + 1j * rng.standard_normal(2 ** L)
    psi /= np.linalg.norm(psi)
    x = torch.from_numpy(psi).cuda()
    for _ in range(3):
        y = H * x
    torch.cuda.synchronize()
    a, c = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(20):
        y = H * x
    c.record()
    torch.cuda.synchronize()
    res = {"D": 2 ** L, "matvec_ms": round(a.elapsed_time(c) / 20, 4)}
    for _ in range(2):
        ev, d = ek.lanczos_e0(H, psi, m=steps)
    res["lanczos150"] = {"seconds": round(d["seconds"], 4), "E0": float(ev[0])}
    o = O.tensor(L)
    Ho = O.operator([O.spin((1.0, "xx"), (1.0, "yy"), (1.5, "zz"))] * (L - 1), inds, o)
    Ho.mul(psi)
    t = time.perf_counter()
    yo = Ho.mul(psi)
    res["cpu_oracle_mul_ms"] = round((time.perf_counter() - t) * 1e3, 3)
    res["cpu_oracle_threads"] = os.cpu_count()
    res["rel_diff_vs_oracle"] = float(np.linalg.norm(y.cpu().numpy() - yo) / np.linalg.norm(yo))
    return res


def config5_ensemble(ek, n_inst=512, seed=2024, steps=200):
    """512 random-field XXZ chains (open, Delta=1, h_i ~ U[-3,3] on spin-1/2 z),
    L drawn from {12,14,16,18,20}, ProjectedBasis N=L/2.  Time to E0 (nev=1)
    and to the four lowest levels (nev=4, for the gap ratio): FP64 batched,
    mixed batched, and FP64 one instance at a time (estimated from a sample)."""
    rng = np.random.default_rng(seed)
    bond = ek.spin((1.0, "xx"), (1.0, "yy"), (1.0, "zz"))
    ops = []
    for _ in range(n_inst):
        Lq = int(rng.choice([12, 14, 16, 18, 20]))
        h = rng.uniform(-3, 3, Lq)
        mats = [bond] * (Lq - 1) + [hi * ek.spin("z") for hi in h]
        inds = [[i, i + 1] for i in range(1, Lq)] + [[i] for i in range(1, Lq + 1)]
        ops.append(ek.operator(mats, inds, ek.ProjectedBasis(L=Lq, N=Lq // 2)))
    rows = sum(op.size(1) for op in ops)
    v0s = [np.random.default_rng(q).standard_normal(op.size(1)) for q, op in enumerate(ops)]
    res = {"instances": n_inst, "rows": rows}
    for nev in (1, 4):
        r, ev = {}, {}
        for name, kw in (("fp64_batched", {}), ("mixed_batched", {"precision": "mixed"})):
            for _ in range(2):
                ev[name], d = ek.batch_lanczos_e0(ops, v0s, m=steps, nev=nev, tol=1e-12,
                                                  check_every=10, **kw)
            r[name] = {"seconds": round(d["seconds"], 4), "max_steps": d["steps"],
                       "max_steps_fp32": d["steps_low"], "seconds_stage1": round(d["seconds_stage1"], 4),
                       "seconds_refine": round(d["seconds_refine"], 4),
                       "matvecs": d["matvecs"]}
        a, b = ev["fp64_batched"], ev["mixed_batched"]
        r["dE0_rel_max_mixed_vs_fp64"] = float(np.max(np.abs(b[:, 0] - a[:, 0]) / np.abs(a[:, 0])))
        r["dE_rel_max_all_levels_mixed_vs_fp64"] = float(np.max(np.abs(b - a) / np.abs(a[:, :1])))
        ns = 32
        t = time.perf_counter()
        for q in range(ns):
            ek.lanczos_e0(ops[q], v0s[q], m=steps, nev=nev, tol=1e-12, check_every=10)
        seq = (time.perf_counter() - t) * n_inst / ns
        r["fp64_one_at_a_time_seconds_est"] = round(seq, 3)
        r["speedup_mixed_batched_vs_fp64_one_at_a_time"] = round(seq / r["mixed_batched"]["seconds"], 2)
        r["speedup_mixed_batched_vs_fp64_batched"] = round(
            r["fp64_batched"]["seconds"] / r["mixed_batched"]["seconds"], 3)
        if nev == 4:
            r["mean_gap_ratio_low4_fp64"] = float(np.mean([np.mean(ek.gapratio(e)) for e in a]))
            r["mean_gap_ratio_low4_mixed"] = float(np.mean([np.mean(ek.gapratio(e)) for e in b]))
        res["E0_nev1" if nev == 1 else "low4_nev4"] = r
    return res


def config4_sectors(ek, steps=100, block=True):
    """Periodic XXZ L=26, Delta=1.5, N=13, all 26 momentum sectors in one batch:
    the lowest 4 eigenvalues per sector (single-vector Lanczos per sector;
    with block=True also the block Lanczos with 64 right-hand sides)."""
    bond = ek.spin((1.0, "xx"), (1.0, "yy"), (1.5, "zz"))
    bases = [ek.TranslationalBasis(L=26, N=13, k=k) for k in range(26)]
    for b in bases:
        b.set_search("rank")  # rank tables (41.6 MB each) for the single-vector runs
    ops = [ek.trans_inv_operator(bond, 2, b) for b in bases]
    res = {"sectors": 26, "dims": [op.size(1) for op in ops], "index_search": "rank"}
    low = {}
    for name, kw in (("fp64_batched", {}), ("mixed_batched", {"precision": "mixed"})):
        for _ in range(2):
            ev, d = ek.batch_lanczos_e0(ops, m=300, nev=4, tol=1e-12, check_every=10, **kw)
        res[name] = {"seconds": round(d["seconds"], 4), "max_steps": d["steps"],
                     "max_steps_fp32": d["steps_low"], "seconds_stage1": round(d["seconds_stage1"], 4),
                     "seconds_refine": round(d["seconds_refine"], 4)}
        res[name + "_low4_k0"] = [float(v) for v in ev[0]]
        low[name] = ev
    res["E0_all_sectors"] = float(np.min(ev[:, 0]))
    res["dE_rel_max_mixed_vs_fp64_low4"] = float(np.max(
        np.abs(low["mixed_batched"] - low["fp64_batched"]) / np.abs(low["fp64_batched"][:, :1])))
    if not block:
        return res
    # the block form: 64 seeded N(0,1) right-hand sides per sector, 100 block steps
    evb, db = ek.block_lanczos(ops, block=64, m=steps, nev=4, check_every=0, seed=2026)
    res["block64_lanczos"] = {k: (round(v, 4) if isinstance(v, float) else v)
                              for k, v in db.items()}
    res["block64_lanczos"]["dE_rel_max_vs_single_vector_fp64"] = float(np.max(
        np.abs(evb - low["fp64_batched"]) / np.abs(low["fp64_batched"][:, :1])))
    return res


def config3_krylov(ek, ntimes=101):
    """J1-J2 XXZ L=32 (J2=0.5), N=16, k=0 (D=18,784,170): Krylov exp(-iHt) psi0
    from a seeded random product state at t = 0, 0.1, ..., 10 (all 101 states
    kept in HBM), m = 30.  FP32 complex Krylov vectors (mixed) against the FP64
    run: worst fidelity and energy drift over the trajectory; both again on the
    materialised operator."""
    import torch
    from edkit_b200 import _lib as E
    b = ek.TranslationalBasis(L=32, N=16, k=0)
    H = ek.trans_inv_operator(ek.spin((1.0, "xx"), (1.0, "yy"), (1.0, "zz")), 2, b) + \
        ek.trans_inv_operator(ek.spin((0.5, "xx"), (0.5, "yy"), (0.5, "zz")), [1, 3], b)
    b.set_search("rank")  # 2.4 GB rank table: the fastest matrix-free search here
    rng = np.random.default_rng(99)
    dg = np.zeros(32, dtype=np.int64)
    dg[rng.choice(32, 16, replace=False)] = 1
    psi0 = torch.from_numpy(ek.productstate(dg, b).astype(np.complex128)).cuda()
    ts = np.round(np.arange(ntimes) * 0.1, 10)
    D = b.size(1)
    res = {"D": D, "times": len(ts)}
    lib = E.load()
    y = torch.empty(D, dtype=torch.complex128, device="cuda")

    def energy(v):
        E.check(lib.edk_apply(H._h, E.C128, E.ptr(v), E.ptr(y), 1, D, D, 0, E.DEVICE))
        return float(torch.vdot(v, y).real / torch.vdot(v, v).real)

    def run(prec):
        psi, d = ek.timeevolve(H, psi0, ts, tol=1e-10, m_init=30, m_max=30,
                               return_diagnostics=True, precision=prec)
        return psi, {"seconds": round(d.seconds, 3), "matvecs": d.matvecs,
                     "restarts": d.restarts}

    def compare(a, m):
        fid = []
        for q in range(a.shape[1]):
            x, z = a[:, q], m[:, q]
            fid.append(float(torch.vdot(x, z).abs() ** 2 /
                             (torch.vdot(x, x).real * torch.vdot(z, z).real)))
        return 1.0 - min(fid)

    e_init = energy(psi0)
    ref, res["fp64"] = run("fp64")
    mix, res["mixed"] = run("mixed")
    res["max_infidelity_mixed_vs_fp64"] = compare(ref, mix)
    res["max_energy_drift_fp64"] = max(abs(energy(ref[:, q].contiguous()) - e_init)
                                       for q in range(0, len(ts), 10))
    res["max_energy_drift_mixed"] = max(abs(energy(mix[:, q].contiguous()) - e_init)
                                        for q in range(0, len(ts), 10))
    del mix
    torch.cuda.empty_cache()
    t = time.perf_counter()
    entries = H.sparse_()
    res["materialized_build_seconds"] = round(time.perf_counter() - t, 3)
    res["materialized_entries"] = entries
    for prec in ("fp64", "mixed"):
        st, res[prec + "_materialized"] = run(prec)
        res[prec + "_materialized"]["max_infidelity_vs_fp64_matrix_free"] = compare(ref, st)
        del st
        torch.cuda.empty_cache()
    H.clear_sparse_cache_()
    return res


def cpu_baseline(balg, D, budget_s=15.0):
    """The oracle's threaded mul (EDKit's column scatter with thread-private
    outputs) on this host's cores: full H*psi products of the same sector,
    repeated for about budget_s / 3 seconds (at least two) after one untimed."""
    import oracle as O
    o = O.translational(L, k=K_MOM, N=N)
    Ho = O.trans_inv_operator(O.spin((1.0, "xx"), (1.0, "yy"), (DELTA, "zz")), 2, o)
    x = np.random.default_rng(1234).standard_normal(D)
    Ho.mul_cols(x, 1, D)
    ts = []
    t_all = time.perf_counter()
    while len(ts) < 2 or (time.perf_counter() - t_all < budget_s / 3 and len(ts) < 50):
        t = time.perf_counter()
        Ho.mul_cols(x, 1, D)
        ts.append(time.perf_counter() - t)
    dt = float(np.mean(ts))
    cores = O.lib().orc_num_threads()
    return {"value": round(balg / dt / 1e9, 6), "unit": "GB/s", "cores": cores,
            "kind": "port",
            "sample": f"{len(ts)} full H*psi products over all {D} columns (EDKit mul: column "
                      f"scatter, thread-private outputs), {dt:.3f} s each"}


def run_reference(args):
    """The reference arm: the C++ restatement of EDKit's threaded mul (column
    scatter over every input column, thread-private outputs summed at the end,
    src/Operator.jl:340-352) on this host's cores.  A step is one full H*psi
    over the sector, the same product the GPU arm times.  When K + W full
    products would not fit in --ref-budget seconds, only as many steps as fit
    are timed (at least 3) and the line says so."""
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
    t = time.perf_counter()
    Ho.mul_cols(x, 1, D)  # first product: page-in and thread start-up, not timed
    per_step = time.perf_counter() - t
    n_fit = int(args.ref_budget / max(per_step, 1e-9))
    warm = max(1, min(args.warmup, max(n_fit - 3, 1)))
    timed = max(3, min(args.steps, n_fit - warm))
    for _ in range(warm):
        Ho.mul_cols(x, 1, D)
    ts = []
    for _ in range(timed):
        t = time.perf_counter()
        Ho.mul_cols(x, 1, D)
        ts.append(time.perf_counter() - t)
    ms = float(np.mean(ts)) * 1e3
    value = balg / (ms * 1e-3) / 1e9
    cores = O.lib().orc_num_threads()
    sample = (f"{timed} of {args.steps} steps timed after {warm} warm-up steps, each one full "
              f"H*psi over all {D} columns (C++ restatement of EDKit mul: column scatter, "
              f"thread-private outputs; Julia is not installed)")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(value, 6), "unit": "GB/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded normal psi)",
        "config": {"workload": WORKLOAD, "D": D, "nnz_hits": nnz,
                   "algorithmic_bytes_per_step": balg,
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
    ap.add_argument("--search", default="rank", choices=["rank", "hash", "sorted"],
                    help="index search of the target rows (rank table, hash table, sorted array)")
    ap.add_argument("--skip-e0", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-materialized", action="store_true")
    ap.add_argument("--extras", action="store_true",
                    help="also run the batched (configs 4, 5) and Krylov (config 3) workloads")
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--ref-budget", type=float, default=120.0,
                    help="seconds of host time the reference arm may spend on its timed steps")
    ap.add_argument("--clock-soak", type=float, default=1.0,
                    help="seconds of untimed steps sampled for clocks before the timed region")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
