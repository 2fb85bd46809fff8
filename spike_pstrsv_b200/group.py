"""Many systems in one captured launch sequence (spk_group_* in
include/spike_pstrsv.h), the partition-count autotuner, and the batched
benchmark over many independent systems.

Benchmark workload (full form): 512 lower-triangular systems with m
log-uniform in [1,024, 262,144], off-diagonals per row ~ Poisson(8) at seeded
positions within a per-system band of 32-256, values N(0,1)/16 with diagonal
1 + sum|off|, k right-hand sides per system drawn from {1, 2, 4, 8, 16, 32};
FP64 and FP32 + FP64 refinement; seeded synthetic data.

    python -m spike_pstrsv_b200.group [--count 512]
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import time

import numpy as np

from . import synth
from .capi import SpkError, System, lib

MODE_FP64 = 0
MODE_FP32_IR = 1

_bound = False


def _bind():
    global _bound
    L = lib()
    if not _bound:
        vp, i, ll = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong
        L.spk_group_create.argtypes = [ctypes.POINTER(vp), i, ctypes.POINTER(vp), ctypes.POINTER(i),
                                       ctypes.POINTER(vp), ctypes.POINTER(ll), ctypes.POINTER(vp),
                                       ctypes.POINTER(ll), i, i, vp]
        L.spk_group_solve.argtypes = [vp, vp]
        L.spk_group_residual.argtypes = [vp, vp, ctypes.POINTER(ctypes.c_double)]
        L.spk_group_info.argtypes = [vp, ctypes.c_char_p]
        L.spk_group_info.restype = ll
        L.spk_group_destroy.argtypes = [vp]
        _bound = True
    return L


def _check(rc):
    if rc != 0:
        raise SpkError(rc, lib().spk_last_error().decode())


class Group:
    """systems: preprocessed capi.System objects; B, X: CUDA tensors of shape
    (nrhs_i, n_i) (row k = right-hand side k); the tensors must stay alive and
    in place while the group is used.  stream: a cudaStream_t handle (not the
    legacy default stream: the launches are captured)."""

    def __init__(self, systems, B, X, mode: int = MODE_FP64, iters: int = 1, stream: int = 0):
        L = _bind()
        n = len(systems)
        self._keep = (systems, B, X)
        hs = (ctypes.c_void_p * n)(*[s.h.value if hasattr(s.h, "value") else s.h for s in systems])
        nr = (ctypes.c_int * n)(*[int(b.shape[0]) for b in B])
        bp = (ctypes.c_void_p * n)(*[b.data_ptr() for b in B])
        lb = (ctypes.c_longlong * n)(*[int(b.stride(0)) for b in B])
        xp = (ctypes.c_void_p * n)(*[x.data_ptr() for x in X])
        lx = (ctypes.c_longlong * n)(*[int(x.stride(0)) for x in X])
        h = ctypes.c_void_p()
        _check(L.spk_group_create(ctypes.byref(h), n, hs, nr, bp, lb, xp, lx, int(mode), int(iters),
                                  ctypes.c_void_p(stream)))
        self.h = h
        self.stream = stream

    def solve(self, stream: int | None = None):
        _check(_bind().spk_group_solve(self.h, ctypes.c_void_p(self.stream if stream is None else stream)))

    def residual(self, stream: int | None = None) -> float:
        w = ctypes.c_double()
        _check(_bind().spk_group_residual(self.h, ctypes.c_void_p(self.stream if stream is None else stream),
                                          ctypes.byref(w)))
        return w.value

    def info(self, name: str) -> int:
        return int(_bind().spk_group_info(self.h, name.encode()))

    def close(self):
        if self.h:
            _bind().spk_group_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- autotuner --------------------------------------------------------------------

ROWS_PER_PARTITION = (256, 512, 1024, 2048, 4096, 8192)


def size_class(m: int) -> int:
    return int(math.floor(math.log2(max(m, 1))))


def partitions_for(m: int, rows: int) -> int:
    return int(max(1, min(1024, m // rows)))


def autotune(mats, nrhs, mode: int = MODE_FP64, candidates=ROWS_PER_PARTITION, reps: int = 5):
    """Rows per Spike partition for each size class (floor(log2 m)): on the
    class's median system with the class's median right-hand-side count, time a
    batched solve for every candidate and keep the fastest.  Returns
    {class: rows_per_partition} and the timing table."""
    import torch
    classes = {}
    for i, L in enumerate(mats):
        classes.setdefault(size_class(L.m), []).append(i)
    choice, table = {}, {}
    stream = torch.cuda.current_stream()
    # the group runs the partition kernels, whose speed the partition count sets;
    # a single system's batched solve would take the chain kernels, which do not
    # depend on it, so the timings force the partition path
    saved = os.environ.get("SPK_CHAIN_BATCH")
    os.environ["SPK_CHAIN_BATCH"] = "0"
    try:
        return _autotune_classes(mats, nrhs, mode, candidates, reps, classes, choice, table, stream)
    finally:
        if saved is None:
            os.environ.pop("SPK_CHAIN_BATCH", None)
        else:
            os.environ["SPK_CHAIN_BATCH"] = saved


def _autotune_classes(mats, nrhs, mode, candidates, reps, classes, choice, table, stream):
    import torch
    for c, idx in sorted(classes.items()):
        idx = sorted(idx, key=lambda i: mats[i].m)
        rep = idx[len(idx) // 2]
        L = mats[rep]
        k = int(np.median([nrhs[i] for i in idx]))
        _, B = synth.make_rhs(L, seed=rep, nrhs=k)
        dB = torch.from_numpy(B).cuda()
        dX = torch.zeros_like(dB)
        best, times = None, {}
        for rows in candidates:
            P = partitions_for(L.m, rows)
            if P in [partitions_for(L.m, r) for r in times]:
                continue  # same partition count as a tried candidate
            S = System().preproc(L.a, L.ia, L.ja, L.m, P, "L", 1)
            S.solve_batch(dB, dX, mode=mode, tol=-1.0, maxit=1, stream=stream.cuda_stream, want_resid=False)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(reps):
                S.solve_batch(dB, dX, mode=mode, tol=-1.0, maxit=1, stream=stream.cuda_stream, want_resid=False)
            torch.cuda.synchronize()
            times[rows] = (time.perf_counter() - t0) / reps
            del S
            if best is None or times[rows] < times[best]:
                best = rows
        choice[c] = best
        table[c] = {"m": L.m, "nrhs": k, "seconds": times}
    return choice, table


# ---- benchmark ----------------------------------------------------------------------

def build(count: int, seed: int = 0, m_lo: int = 1024, m_hi: int = 262144, band_lo: int = 32, band_hi: int = 256):
    pool = synth.batch_pool(count, m_lo=m_lo, m_hi=m_hi, band_lo=band_lo, band_hi=band_hi, seed=seed)
    mats = [p[0] for p in pool]
    nrhs = [p[1] for p in pool]
    rhs = [synth.make_rhs(L, seed=seed + 7 * i + 1, nrhs=k) for i, (L, k) in enumerate(zip(mats, nrhs))]
    return mats, nrhs, rhs


def run(count: int = 512, reps: int = 5, seed: int = 0, tune: bool = True, m_hi: int = 262144):
    import torch
    mats, nrhs, rhs = build(count, seed, m_hi=m_hi)
    dev = torch.device("cuda")
    stream = torch.cuda.Stream()
    out = {"systems": count, "sum_rows": int(sum(L.m for L in mats)), "sum_nnz": int(sum(L.nnz for L in mats)),
           "rhs": int(sum(nrhs)), "modes": []}
    choice, table = autotune(mats, nrhs) if tune else ({}, {})
    out["autotune"] = {str(c): {"rows_per_partition": r, **table[c]} for c, r in choice.items()}
    systems = []
    t0 = time.perf_counter()
    for L in mats:
        rows = choice.get(size_class(L.m), 4096)
        systems.append(System().preproc(L.a, L.ia, L.ja, L.m, partitions_for(L.m, rows), "L", 1))
    out["preprocess_s"] = time.perf_counter() - t0
    B = [torch.from_numpy(b).to(dev) for _, b in rhs]
    # plain FP64 one solve per call (device-resident), per system
    t_plain = []
    x1 = [torch.zeros(L.m, dtype=torch.float64, device=dev) for L in mats]
    with torch.cuda.stream(stream):
        sp = stream.cuda_stream
        for S, b, x in zip(systems, B, x1):
            S.solve_device(b[0].data_ptr(), x.data_ptr(), sp)
        stream.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            for S, b, x, k in zip(systems, B, x1, nrhs):
                for _ in range(k):
                    S.solve_device(b[0].data_ptr(), x.data_ptr(), sp)
        e1.record(stream)
        stream.synchronize()
    plain_s = e0.elapsed_time(e1) / 1e3 / reps
    out["plain_fp64_solves_per_s"] = sum(nrhs) / plain_s
    for mode in (MODE_FP64, MODE_FP32_IR):
        X = [torch.zeros_like(b) for b in B]
        iters = 0 if mode == MODE_FP64 else 1
        g = Group(systems, B, X, mode=mode, iters=iters, stream=stream.cuda_stream)
        g.solve()
        stream.synchronize()
        res = g.residual()
        if mode == MODE_FP32_IR and res > 1e-12:
            iters = 2
            g.close()
            g = Group(systems, B, X, mode=mode, iters=iters, stream=stream.cuda_stream)
            g.solve()
            res = g.residual()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            g.solve()
        e1.record(stream)
        stream.synchronize()
        ms = e0.elapsed_time(e1) / reps
        err = 0.0
        for (Xt, _), x in zip(rhs, X):
            xx = x.cpu().numpy()
            err = max(err, float(np.abs(xx - Xt).max() / np.abs(Xt).max()))
        out["modes"].append({"mode": "fp64" if mode == MODE_FP64 else "fp32_ir", "refinement_steps": iters,
                             "ms_per_group_solve": ms, "solves_per_s": sum(nrhs) * 1e3 / ms,
                             "vs_plain_fp64": sum(nrhs) * 1e3 / ms / out["plain_fp64_solves_per_s"],
                             "scaled_residual": res, "max_rel_err_vs_x_true": err,
                             "graph_kernels": g.info("kernels"), "task_items": g.info("task_items"),
                             "virtual_systems": g.info("virtual_systems")})
        g.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--count", type=int, default=512)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--no-tune", action="store_true")
    args = ap.parse_args()
    print(json.dumps(run(args.count, args.reps, tune=not args.no_tune)))


if __name__ == "__main__":
    main()
