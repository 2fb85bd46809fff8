#!/usr/bin/env python
"""Headline benchmark: Spike sparse triangular solves per second on one B200.

Workload: the large banded lower-triangular system (m = 4,194,304 rows, each row
16 off-diagonals at distinct columns among the 64 preceding ones, values
N(0,1)/16, diagonal 1 + sum|off|; nnz = 71,303,032; FP64 values, int32 indices;
one right-hand side b = L x_true), solved with uplo='L' and nthreads = 1024
Spike partitions.  Seeded synthetic data stands in for the reference's external
MatrixMarket files.

A step is one solve (spike_pstrsv_solve) of that system.
  value  : solves/s with b and x resident in HBM, device-timed with CUDA events
           on the solve's stream over --steps solves (the 0.94 GB matrix is
           larger than the 126 MB L2, so no flush is needed between steps).
  e2e    : solves/s through the reference-facing C ABI (spike_pstrsv_solve)
           with pinned host buffers: every step copies b host->device and x
           device->host inside the timed region.
  roofline: the algorithmic bytes of one solve, B = 12 nnz + 4 (m+1) + 16 m
           (each matrix byte once; the second pass over the coupled rows is not
           credited), over the solve kernels' event-timed duration per solve,
           against the measured HBM copy bandwidth.  kernel_rows_gbs credits
           B/m per row each launch solves (rows solved twice count twice).
  sweep  : the same workload at 16/64/256/1024 partitions, uplo L and U, with
           spike truncation (default) and in exact mode (the reference's
           phases: D1 sweep, reduced system, D2 sweep).
  latency: the small Poisson 128x128 system at 4 partitions.
  cpu_baseline: the reference's own OpenMP code (oracle/_ref, built from the
           reference sources) on a bounded sample of the same workload.

--impl reference times the reference's OpenMP solve of the same workload on the
host cores (rank 0 only under torchrun).

Multi-GPU: one process per GPU, each solving its own copy of the system (the
path partitions into independent systems; no collective on the data path),
timed as the max over ranks; value = total solves of all ranks / that time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "solves/s & HBM GB/s at resid≤1e-12: batched/served vs plain FP64; p50/p99 lat"
M_FULL = 4194304


def alg_bytes(m: int, nnz: int) -> int:
    return 12 * nnz + 4 * (m + 1) + 16 * m


def max_over_ranks(x: float, device, world: int) -> float:
    """The largest of every rank's x (one all-reduce; the timing rule of the
    multi-GPU replicas: the job takes as long as its slowest rank)."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replicas_value(ms_max: float, world: int) -> float:
    """Whole-job solves/s of `world` replicas that each solve once per step."""
    return world * 1e3 / ms_max


def batched_bytes(m: int, nnz: int, k: int, mode: int, iters: int) -> int:
    """Algorithmic bytes of one batch of k right-hand sides: FP64 solve
    12 nnz + 4 (m+1) + 16 k m; FP32 solve 8 nnz + 4 (m+1) + 16 k m, plus per
    refinement step an FP64 residual (12 nnz + 4 (m+1) + 24 k m) and an FP32
    correction solve."""
    if mode == 0:
        return 12 * nnz + 4 * (m + 1) + 16 * k * m
    solve32 = 8 * nnz + 4 * (m + 1) + 16 * k * m
    resid = 12 * nnz + 4 * (m + 1) + 24 * k * m
    return solve32 + iters * (resid + solve32)


def run_batched(S, L, x_true_k, dev, stream, k: int, mode: int, steps: int, warmup: int):
    """Batches of k right-hand sides through spk_solve_batch (FP64, or FP32 +
    FP64 refinement with the step count a checked run needs for scaled residual
    <= 1e-12), device-timed with CUDA events over `steps` batches."""
    import torch
    from spike_pstrsv_b200 import synth
    m, nnz = L.m, L.nnz
    Xt, Bk = synth.make_rhs(L, seed=1, nrhs=k)
    dB = torch.from_numpy(Bk).to(dev)
    dX = torch.zeros_like(dB)
    sp = stream.cuda_stream
    iters, _ = S.solve_batch(dB, dX, mode=mode, tol=1e-12, maxit=8, stream=sp)
    for _ in range(warmup):
        S.solve_batch(dB, dX, mode=mode, tol=-1.0, maxit=iters, stream=sp, want_resid=False)
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    l0 = S.scalar("launches")
    e0.record(stream)
    for _ in range(steps):
        S.solve_batch(dB, dX, mode=mode, tol=-1.0, maxit=iters, stream=sp, want_resid=False)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    launches = S.scalar("launches") - l0
    ms = e0.elapsed_time(e1) / steps
    _, resid = S.solve_batch(dB, dX, mode=mode, tol=-1.0, maxit=iters, stream=sp)
    X = dX.cpu().numpy()
    err = max(float(np.linalg.norm(X[i] - Xt[i]) / np.linalg.norm(Xt[i])) for i in range(k))
    nb = batched_bytes(m, nnz, k, mode, iters)
    return {"mode": "fp64" if mode == 0 else "fp32_ir", "rhs_per_batch": k, "refinement_steps": iters,
            "ms_per_batch": ms, "solves_per_s": k * 1e3 / ms, "hbm_gbs": nb / (ms * 1e-3) / 1e9,
            "algorithmic_bytes_per_batch": nb, "scaled_residual": resid, "rel_err_vs_x_true": err,
            "gpu_launches_per_batch": launches / steps}


def node0_cpus():
    """CPUs of NUMA node 0 (sysfs), for pinning the reference's OpenMP threads the
    way its experiment script pins them to one node."""
    try:
        txt = open("/sys/devices/system/node/node0/cpulist").read().strip()
    except OSError:
        return None
    cpus = set()
    for part in txt.split(","):
        if "-" in part:
            a, b = part.split("-")
            cpus.update(range(int(a), int(b) + 1))
        elif part:
            cpus.add(int(part))
    return sorted(cpus)


def kernel_time_per_solve(S, db, dx, sp, dev, n):
    """Per-phase device time of n solves (events on the solve stream), ms per solve."""
    import torch
    S.set_profiling(True)
    for _ in range(n):
        S.solve_device(db.data_ptr(), dx.data_ptr(), sp)
    torch.cuda.synchronize(dev)
    ph, nsol = S.phase_times()
    S.set_profiling(False)
    return [p / max(nsol, 1) for p in ph]


def timed_solves(S, db, dx, sp, stream, dev, warmup, steps):
    import torch
    for _ in range(warmup):
        S.solve_device(db.data_ptr(), dx.data_ptr(), sp)
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        S.solve_device(db.data_ptr(), dx.data_ptr(), sp)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    S.check()
    return e0.elapsed_time(e1) / steps


def run_sweep(L, dev, stream, peak, steps: int = 30):
    """Every partition count and uplo of the banded workload, default (spike
    truncation) and exact mode, device-resident, CUDA-event timed."""
    import torch
    import spike_pstrsv_b200 as spk
    from spike_pstrsv_b200 import synth
    B = alg_bytes(L.m, L.nnz)
    sp = stream.cuda_stream
    out = []
    for uplo in ("L", "U"):
        A = L if uplo == "L" else synth.transpose(L)
        x_true, b = synth.make_rhs(A, seed=0)
        db = torch.from_numpy(b).to(dev)
        dx = torch.zeros_like(db)
        for P in (16, 64, 256, 1024):
            t0 = time.perf_counter()
            S = spk.System().preproc(A.a, A.ia, A.ja, A.m, P, uplo, 1)
            pre_s = time.perf_counter() - t0
            for exact in (False, True):
                if exact:
                    S.set_truncation(-1.0)
                n = steps if not exact else max(3, steps // 6)
                ms = timed_solves(S, db, dx, sp, stream, dev, 3, n)
                x = dx.cpu().numpy()
                cell = {"uplo": uplo, "partitions": P, "mode": "exact" if exact else "default",
                        "solves_per_s": 1e3 / ms, "ms_per_solve": ms,
                        "frac": B / (ms * 1e-3) / 1e9 / peak,
                        "scaled_residual": scaled_residual(A, x, b),
                        "rel_err_vs_x_true": float(np.linalg.norm(x - x_true) / np.linalg.norm(x_true)),
                        "solver": "chain" if S.scalar("chain") else "partition",
                        "launches_per_solve": S.scalar("launches_per_solve")}
                if exact:
                    cell["reduced_rows_kept"] = S.scalar("kept_reduced_rows")
                    ph = kernel_time_per_solve(S, db, dx, sp, dev, n)
                    cell["phases_ms"] = {"d1_local": ph[0], "reduced": ph[1], "d2_coupled": ph[2]}
                else:
                    cell["preprocess_s"] = pre_s
                    cell["chains"] = S.scalar("chains")
                out.append(cell)
            S.close()
            del S
            torch.cuda.empty_cache()
    return out


def run_latency(dev, stream, steps: int = 200):
    """The small Poisson 128x128 lower-triangular system (m = 16,384) at 4
    partitions: device time per solve back to back, and the wall time of one
    synchronous call with host arrays."""
    import torch
    import spike_pstrsv_b200 as spk
    from spike_pstrsv_b200 import synth
    L = synth.poisson2d_lower(128)
    x_true, b = synth.make_rhs(L, seed=0)
    S = spk.System().preproc(L.a, L.ia, L.ja, L.m, 4, "L", 1)
    db = torch.from_numpy(b).to(dev)
    dx = torch.zeros_like(db)
    ms = timed_solves(S, db, dx, stream.cuda_stream, stream, dev, 10, steps)
    x = np.zeros(L.m)
    walls = []
    for k in range(steps // 2 + 10):
        t0 = time.perf_counter()
        S.solve(b, x)
        if k >= 10:
            walls.append(time.perf_counter() - t0)
    walls.sort()
    out = {"workload": "Poisson 128x128 lower triangle, m=16384, nnz=48896, uplo=L, 4 partitions",
           "device_us_per_solve": ms * 1e3,
           "host_call_us_p50": 1e6 * walls[len(walls) // 2],
           "host_call_us_p99": 1e6 * walls[int(0.99 * (len(walls) - 1))],
           "rel_err_vs_x_true": float(np.linalg.norm(x - x_true) / np.linalg.norm(x_true)),
           "solver": "chain" if S.scalar("chain") else "partition"}
    S.close()
    return out


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def scaled_residual(L, x, b):
    from spike_pstrsv_b200 import synth
    r = b - synth.spmv(L, x)
    rowsum = np.add.reduceat(np.abs(L.a), L.ia[:-1].astype(np.int64))
    return float(np.abs(r).max() / (rowsum.max() * np.abs(x).max() + np.abs(b).max()))


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 100 ms while running."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = os.path.join("/tmp", f"spk_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def cpu_baseline_sample(P_full: int, budget_s: float = 12.0):
    """The reference's OpenMP solve on a bounded sample of the workload: the same
    generator at 1/16 of the rows with the same rows per partition, scaled back
    to the full size by the row count (the solve is linear in m)."""
    import oracle
    from spike_pstrsv_b200 import synth
    m_s = M_FULL // 16
    P_s = max(1, P_full // 16)
    L = synth.banded_lower(m_s, seed=0)
    _, b = synth.make_rhs(L, seed=0)
    if oracle.Reference.available():
        R = oracle.Reference()
        R.preproc(synth.mirror(L), P_s, flb=1)
        bu = b[::-1].copy()
        R.solve(bu)
        times = []
        t_end = time.perf_counter() + budget_s
        while time.perf_counter() < t_end or len(times) < 5:
            t0 = time.perf_counter()
            R.solve(bu)
            times.append(time.perf_counter() - t0)
            if len(times) >= 400:
                break
        per = statistics.median(times)
        kind, threads = "reference", P_s
    else:
        times = []
        t_end = time.perf_counter() + budget_s
        while time.perf_counter() < t_end or len(times) < 3:
            t0 = time.perf_counter()
            oracle.sequential_solve(L, b, "L")
            times.append(time.perf_counter() - t0)
        per = statistics.median(times)
        kind, threads = "port", 1
    full = per * (M_FULL / m_s)
    return {"value": 1.0 / full, "unit": "solves/s", "cores": min(threads, os.cpu_count() or 1),
            "threads": threads, "host_cores": os.cpu_count(), "kind": kind,
            "sample": f"banded m={m_s} (1/16 of the rows), uplo=L, nthreads={P_s} (same 4096 rows per "
                      f"partition), median of {len(times)} solves = {per*1e3:.2f} ms, scaled x16 to m={M_FULL}"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import oracle
    from spike_pstrsv_b200 import synth
    if not oracle.Reference.available():
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/libspike_ref.so (the reference sources built here) is missing"}))
        return 0
    cpus = node0_cpus()
    pin = "none"
    if cpus and hasattr(os, "sched_setaffinity"):
        # one NUMA node, as the reference's experiment script pins with numactl
        # (numactl itself is not installed; memory placement is left to first touch)
        os.sched_setaffinity(0, cpus)
        pin = f"node0 cpus {cpus[0]}-{cpus[-1]} ({len(cpus)}) via sched_setaffinity"
    L = synth.banded_lower(M_FULL, seed=0)
    _, b = synth.make_rhs(L, seed=0)
    U = synth.mirror(L)
    bu = b[::-1].copy()
    # the single-core sequential substitution (the profiler's udsol/ldsol baseline)
    seq = []
    for _ in range(3):
        t0 = time.perf_counter()
        oracle.sequential_solve(L, b, "L")
        seq.append(time.perf_counter() - t0)
    R = oracle.Reference()
    t0 = time.perf_counter()
    R.preproc(U, args.P, flb=1)
    pre_s = time.perf_counter() - t0
    pad = 16
    bb = np.zeros(M_FULL + 2 * pad)
    xx = np.zeros(M_FULL + 2 * pad)
    baddr, xaddr = bb.ctypes.data + 8 * pad, xx.ctypes.data + 8 * pad
    times = []
    for k in range(args.warmup + args.steps):
        bb[pad:pad + M_FULL] = bu          # b is clobbered by the reference: re-copied outside the timer
        xx[:] = 0.0
        t0 = time.perf_counter()
        R.solve_raw(baddr, xaddr, timed=False)
        dt = time.perf_counter() - t0
        if k >= args.warmup:
            times.append(dt)
    x = xx[pad:pad + M_FULL][::-1].copy()
    total = sum(times)
    value = len(times) / total
    res = scaled_residual(L, x, b)
    out = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": 1e3 * total / len(times), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "impl": "reference",
           "data": "synthetic banded lower-triangular CSR (seeded), see config",
           "config": {"workload": f"banded lower-triangular m={M_FULL} nnz={L.nnz} uplo=L nthreads={args.P}, "
                                  "reference OpenMP spike_pstrsv_solve via the J L J mirror on its 'U' path",
                      "m": M_FULL, "nnz": int(L.nnz), "partitions": args.P, "uplo": "L"},
           "cpu_baseline": {"value": value, "unit": "solves/s", "cores": min(args.P, os.cpu_count() or 1),
                            "threads": args.P, "host_cores": os.cpu_count(), "kind": "reference",
                            "sample": f"full workload, {len(times)} timed solves after {args.warmup} warm-up, "
                                      f"b re-copied outside the timer; preprocessing {pre_s:.1f} s untimed"},
           "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
           "pinning": pin,
           "sequential_1core": {"solves_per_s": 1.0 / min(seq), "ms_per_solve": 1e3 * min(seq),
                                "what": "forward substitution, one thread (the profiler's ldsol comparator), best of 3"},
           "accuracy": {"scaled_residual": res}}
    print(json.dumps(out))
    return 0


def run_ours(args):
    import torch
    import torch.distributed as dist

    import spike_pstrsv_b200 as spk
    from spike_pstrsv_b200 import synth

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=dev)

    L = synth.banded_lower(M_FULL, seed=0)
    x_true, b = synth.make_rhs(L, seed=0)
    m, nnz = L.m, L.nnz
    B = alg_bytes(m, nnz)

    S = spk.System().preproc(L.a, L.ia, L.ja, m, args.P, "L", 1)
    db = torch.from_numpy(b).to(dev)
    dx = torch.zeros_like(db)
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream

    clocks = ClockSampler(local)
    clocks.start()
    for _ in range(args.warmup):
        S.solve_device(db.data_ptr(), dx.data_ptr(), sp)
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    launches0 = S.scalar("launches")
    e0.record(stream)
    for _ in range(args.steps):
        S.solve_device(db.data_ptr(), dx.data_ptr(), sp)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    launches = S.scalar("launches") - launches0
    S.check()
    ms = e0.elapsed_time(e1) / args.steps
    ms_max = max_over_ranks(ms, dev, world)
    value = replicas_value(ms_max, world)

    # the solve's kernels, event-timed per phase on the solve stream
    ph = kernel_time_per_solve(S, db, dx, sp, dev, args.steps)
    chain = S.scalar("chain") == 1
    if chain:
        rows1, rows4 = S.scalar("chain_rows_phase1"), S.scalar("chain_rows_phase4")
        kernel = "k_chain_solve (phase 1 chain-local sweep + phase 4 re-solve of the coupled rows), 2 launches per solve"
    else:
        rows1, rows4 = S.scalar("rows_phase1"), S.scalar("rows_phase4")
        kernel = "k_tile_solve (phase 1 D1 sweep + phase 3/4 coupled D2 sweep), 2 launches per solve"
    kernel_ms = ph[0] + ph[1] + ph[2]
    peak, peak_kind = peaks()
    achieved = B / (kernel_ms * 1e-3) / 1e9
    kernel_rows_gbs = (B / m) * (rows1 + rows4) / (kernel_ms * 1e-3) / 1e9
    traffic = None
    tp = os.path.join(ROOT, "profiles", "chain_solve_traffic.json" if chain else "tile_solve_traffic.json")
    if os.path.exists(tp):
        with open(tp) as f:
            tr = json.load(f)
        # DRAM bytes per launch, scaled from the ncu capture of the same kernel by
        # the rows each launch solves (traffic grows with the rows)
        traffic = (tr["phase1_dram_bytes_per_row"] * rows1 + tr["phase4_dram_bytes_per_row"] * rows4) / 2 / 1e9

    # end to end through the reference-facing C ABI with pinned host buffers
    bh = torch.from_numpy(b).pin_memory()
    xh = torch.zeros(m, dtype=torch.float64).pin_memory()
    bn, xn = bh.numpy(), xh.numpy()
    spk.spike_pstrsv_preproc(L.a, L.ia, L.ja, m, args.P, "L")
    for _ in range(max(3, args.warmup // 4)):
        spk.spike_pstrsv_solve("L", m, bn, xn, args.P)
    if world > 1:
        dist.barrier()
    n_e2e = max(10, args.steps // 4)
    t0 = time.perf_counter()
    for _ in range(n_e2e):
        spk.spike_pstrsv_solve("L", m, bn, xn, args.P)
    e2e_s = (time.perf_counter() - t0) / n_e2e
    e2e_value = world / max_over_ranks(e2e_s, dev, world)

    # batched forms of the same system (32 right-hand sides per batch)
    nb_steps = max(10, args.steps // 8)
    batched = [run_batched(S, L, None, dev, stream, 32, mode, nb_steps, 3) for mode in (0, 1)]
    for bt in batched:
        bt["vs_plain_fp64"] = bt["solves_per_s"] / value * world
    # served form: Poisson-arrival request stream through the serving loop
    # (reduced pool; python -m spike_pstrsv_b200.serve_bench --full runs the full one)
    served = None
    if world == 1 and not args.no_served:
        from spike_pstrsv_b200 import serve_bench
        served = serve_bench.run(full=False, rates=(50.0, 500.0), nreq=300)
    # many independent systems in one captured launch sequence (reduced pool of
    # 128 systems; python -m spike_pstrsv_b200.group runs the 512-system form)
    systems = None
    if world == 1 and not args.no_served:
        from spike_pstrsv_b200 import group
        systems = group.run(count=128, reps=5)
    sweep = latency = None
    if world == 1 and not args.no_sweep:
        sweep = run_sweep(L, dev, stream, peak)
        latency = run_latency(dev, stream)
    clk = clocks.stop()

    x = dx.cpu().numpy()
    res = scaled_residual(L, x, b)
    err_true = float(np.linalg.norm(x - x_true) / np.linalg.norm(x_true))
    err_e2e = float(np.linalg.norm(xn - x) / np.linalg.norm(x))

    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f64",
               "data": "synthetic: seeded banded lower-triangular CSR standing in for the reference's "
                       "external .mtx files (see config)",
               "config": {"workload": f"banded lower-triangular m={m} nnz={nnz} (16 of the 64 preceding "
                                      f"columns per row), uplo=L, nthreads(partitions)={args.P}, plain FP64 "
                                      "Spike drop-in, 1 RHS per solve",
                          "m": m, "nnz": int(nnz), "partitions": args.P, "uplo": "L", "mode": "plain_fp64",
                          "truncation_tol": 2.0 ** -60,
                          "l2": "inputs larger than L2 (0.94 GB CSR vs 126 MB L2); no flush between steps",
                          "per_gpu": "each rank solves its own copy (weak scaling)"},
               "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                            "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                            "kernel": kernel,
                            "achieved_is": "algorithmic bytes of one solve (12 nnz + 4 (m+1) + 16 m, each matrix "
                                           "byte once) / event-timed kernel time per solve",
                            "traffic_unit": "GB per launch (ncu DRAM bytes per row x rows, averaged over the 2 launches)",
                            "algorithmic_bytes_per_solve": B,
                            "kernel_ms_per_solve": kernel_ms,
                            "kernel_rows_gbs": kernel_rows_gbs,
                            "whole_solve_gbs": B / (ms_max * 1e-3) / 1e9,
                            "whole_solve_frac": B / (ms_max * 1e-3) / 1e9 / peak},
               "phases_ms": {"phase1": ph[0], "reduced": ph[1], "phase4": ph[2],
                             "rows_phase1": rows1, "rows_phase4": rows4, "solver": "chain" if chain else "partition",
                             "chains": S.scalar("chains")},
               "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": 8 * m,
                       "d2h_bytes_per_step": 8 * m, "api": "spike_pstrsv_solve (C ABI), pinned host b/x"},
               "gpu_launches": int(launches),
               "batched": batched,
               "served": served,
               "batched_systems": systems,
               "sweep": sweep,
               "latency_small": latency,
               "clocks": clk,
               "accuracy": {"scaled_residual": res, "rel_err_vs_x_true": err_true,
                            "e2e_vs_device_rel_diff": err_e2e}}
        if world == 1:
            out["cpu_baseline"] = cpu_baseline_sample(args.P)
        print(json.dumps(out))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--P", type=int, default=1024, help="nthreads = Spike partitions")
    ap.add_argument("--no-served", action="store_true", help="skip the serving-loop stream")
    ap.add_argument("--no-sweep", action="store_true", help="skip the partition/uplo/exact sweep and latency")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
