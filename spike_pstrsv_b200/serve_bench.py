"""Serving benchmark: a Poisson-arrival request stream against a pool of resident
matrices, through the serving loop (spike_pstrsv_b200.serve).

Workload (full form): 64 banded lower-triangular matrices with m log-uniform
in [10,000, 2,000,000], off-diagonals per row ~ Poisson(8) within a per-matrix
band of 32-128 (values N(0,1)/16, diagonal 1 + sum|off|), partitions = m / 4096
clamped to [4, 1024]; 95 % of requests solve 1-16 right-hand sides (host
arrays) on a registered matrix, 5 % upload a matrix (a fresh registration,
preprocessed by its first solve); FP32 + FP64 refinement to scaled residual
<= 1e-12; a 40 GB HBM budget with LRU eviction.  Seeded synthetic matrices.

For each offered rate the stream submits requests at exponential intervals from
one client thread while another collects them; reported are the achieved
solves/s (right-hand sides completed / wall time from the first submit to the
last result), p50/p99 request latency (submit to result in host memory; all
requests, uploads with their registration time, and solve requests alone) and
the server's batching and residency counters.  The comparison is the plain
FP64 path, one solve per call with host arrays (spk_solve), on the same request
mix: solves/s = right-hand sides / the sum of their per-matrix solve times.

    python -m spike_pstrsv_b200.serve_bench [--full] [--rates 50,150,500,2000] [--mode fp32ir|fp64]
"""
from __future__ import annotations

import argparse
import json
import threading
import time

import numpy as np

from . import serve, synth
from .capi import System


def partitions(m: int) -> int:
    return int(min(1024, max(4, m // 4096)))


def build_pool(count: int, m_lo: int, m_hi: int, band_lo: int = 32, band_hi: int = 128, seed: int = 0,
               pool_rhs: int = 16):
    rng = np.random.default_rng(seed)
    ms = np.exp(rng.uniform(np.log(m_lo), np.log(m_hi), size=count)).astype(np.int64)
    bands = rng.integers(band_lo, band_hi + 1, size=count)
    pool = []
    for i in range(count):
        L = synth.poisson_banded_lower(int(ms[i]), 8.0, int(bands[i]), seed=10_000 + i)
        Xt, B = synth.make_rhs(L, seed=20_000 + i, nrhs=pool_rhs)
        pool.append({"L": L, "P": partitions(L.m), "X": Xt, "B": B, "band": int(bands[i])})
    return pool


def plain_times(pool, reps: int = 3):
    """Seconds per plain FP64 solve (spk_solve, host arrays) for each matrix."""
    out = []
    for p in pool:
        L = p["L"]
        S = System().preproc(L.a, L.ia, L.ja, L.m, p["P"], "L", 1)
        x = np.zeros(L.m)
        S.solve(p["B"][0], x)
        t0 = time.perf_counter()
        for r in range(reps):
            S.solve(p["B"][r % len(p["B"])], x)
        out.append((time.perf_counter() - t0) / reps)
        S.close() if hasattr(S, "close") else None
        del S
    return np.asarray(out)


def run_stream(pool, rate: float, nreq: int, budget: int, slots: int, mode: int, seed: int,
               upload_frac: float = 0.05):
    rng = np.random.default_rng(seed)
    n_pool = len(pool)
    upload_ids = list(range(n_pool, n_pool + 8))
    plan = []
    for j in range(nreq):
        if rng.random() < upload_frac:
            plan.append(("upload", int(rng.integers(n_pool)), 1))
        else:
            plan.append(("solve", int(rng.integers(n_pool)), int(rng.integers(1, 17))))
    gaps = rng.exponential(1.0 / rate, size=nreq)
    with serve.Server(budget, slots=slots) as S:
        for i, p in enumerate(pool):
            L = p["L"]
            S.put_matrix(i, L.a, L.ia, L.ja, L.m, p["P"], "L")
        # warm: every pool matrix preprocessed once before the stream
        for i, p in enumerate(pool):
            S.submit(i, p["B"][:1], mode).wait()
        tickets = [None] * nreq
        meta = [None] * nreq
        done = threading.Event()
        results = [None] * nreq

        def collect():
            for j in range(nreq):
                while tickets[j] is None:
                    time.sleep(0)
                try:
                    results[j] = tickets[j].wait()
                except Exception as e:  # a failed request is counted, the stream goes on
                    results[j] = e
            done.set()

        th = threading.Thread(target=collect)
        th.start()
        t_start = time.perf_counter()
        t_next = t_start
        up_i = 0
        for j, (kind, src, k) in enumerate(plan):
            t_next += gaps[j]
            dt = t_next - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            p = pool[src]
            if kind == "upload":
                mid = upload_ids[up_i % len(upload_ids)]
                up_i += 1
                L = p["L"]
                t0 = time.perf_counter()
                try:
                    S.put_matrix(mid, L.a, L.ia, L.ja, L.m, p["P"], "L")
                except Exception:
                    mid = src  # the upload slot is still busy: solve on the pool copy
                upload_s = time.perf_counter() - t0
                meta[j] = (src, 1, upload_s)
                tickets[j] = S.submit(mid, p["B"][:1], mode)
            else:
                meta[j] = (src, k, 0.0)
                tickets[j] = S.submit(src, p["B"][:k], mode)
        done.wait()
        th.join()
        t_end = time.perf_counter()
        stats = S.stats()
    failed = [j for j, r in enumerate(results) if isinstance(r, Exception)]
    errors = sorted({str(results[j]) for j in failed})[:3]
    keep = [j for j in range(nreq) if j not in set(failed)]
    results = [results[j] for j in keep]
    meta = [meta[j] for j in keep]
    plan = [plan[j] for j in keep]
    lat = np.array([r.latency_s + m[2] for r, m in zip(results, meta)])
    solve_lat = np.array([r.latency_s for r, m, p in zip(results, meta, plan) if p[0] == "solve"])
    rhs = sum(m[1] for m in meta)
    worst_res = max(r.scaled_residual for r in results)
    err = 0.0
    wrong = []
    for r, m, pl in zip(results, meta, plan):
        Xt = pool[m[0]]["X"][:m[1]]
        e = float(np.abs(r.x - Xt).max() / np.abs(Xt).max())
        err = max(err, e)
        if e > 1e-10:
            wrong.append({"matrix": m[0], "m": pool[m[0]]["L"].m, "kind": pl[0], "rhs": m[1],
                          "batch_rhs": r.batch_rhs, "resid": r.scaled_residual, "steps": r.refinement_steps,
                          "rel_err": e})
    wall = t_end - t_start
    return {"offered_req_per_s": rate, "requests": nreq, "failed": len(failed), "failures": errors,
            "rhs": int(rhs), "wall_s": wall,
            "solves_per_s": rhs / wall, "p50_ms": float(np.percentile(lat, 50) * 1e3),
            "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "solve_p50_ms": float(np.percentile(solve_lat, 50) * 1e3),
            "solve_p99_ms": float(np.percentile(solve_lat, 99) * 1e3), "mean_batch_rhs": stats["rhs_batched"] / max(stats["batches"], 1),
            "uploads": sum(1 for p in plan if p[0] == "upload"), "max_scaled_residual": worst_res,
            "max_rel_err_vs_x_true": err, "wrong_results": wrong[:20], "n_wrong": len(wrong), "server": stats, "plan": [(m[0], m[1]) for m in meta]}


def run(full: bool = False, rates=(50.0, 150.0, 500.0, 2000.0), nreq: int | None = None, slots: int = 4, seed: int = 0,
        mode: int = serve.MODE_FP32_IR):
    if full:
        pool = build_pool(64, 10_000, 2_000_000, seed=seed)
        budget = 40 << 30
        nreq = nreq or 2000
        desc = "64 matrices, m log-uniform [1e4, 2e6], band 32-128, 40 GB budget"
    else:
        pool = build_pool(16, 10_000, 500_000, seed=seed)
        budget = 8 << 30
        nreq = nreq or 600
        desc = "16 matrices, m log-uniform [1e4, 5e5], band 32-128, 8 GB budget (reduced form)"
    tp = plain_times(pool)
    runs = []
    for rate in rates:
        r = run_stream(pool, rate, nreq, budget, slots, mode, seed + int(rate))
        plan = r.pop("plan")
        plain_s = sum(k * tp[src] for src, k in plan)
        r["plain_fp64_solves_per_s"] = r["rhs"] / plain_s
        r["vs_plain_fp64"] = r["solves_per_s"] / r["plain_fp64_solves_per_s"]
        runs.append(r)
    return {"workload": desc, "mode": "fp32_ir" if mode == serve.MODE_FP32_IR else "fp64", "slots": slots,
            "sum_rows": int(sum(p["L"].m for p in pool)), "runs": runs}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--full", action="store_true")
    ap.add_argument("--rates", default="50,150,500,2000")
    ap.add_argument("--requests", type=int, default=None)
    ap.add_argument("--slots", type=int, default=4)
    ap.add_argument("--mode", default="fp32ir", choices=["fp32ir", "fp64"])
    args = ap.parse_args()
    mode = serve.MODE_FP32_IR if args.mode == "fp32ir" else serve.MODE_FP64
    out = run(args.full, [float(r) for r in args.rates.split(",")], args.requests, args.slots, mode=mode)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
