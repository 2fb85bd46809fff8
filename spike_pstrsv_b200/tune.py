"""Per-system autotuner of the chain solver (spk_tune).

The one-right-hand-side solve has two knobs: rows per chain task (the plan's
chain length; fewer rows give more tasks but a larger share of re-solved coupled
rows) and the staging depth of its kernel (2 or 3 tiles in flight).  The batched
solve has two more: its path (chain kernels or the partition kernels) and its
own rows per chain task.  Each candidate is timed with CUDA events on the
system's own solves of the caller's right-hand sides, and the fastest setting of
each knob is kept (rows and stages jointly, then path and batch rows jointly).
The reference has no counterpart: its only knob is the thread count.
"""
from __future__ import annotations


def _events_ms(fn, stream, reps: int, warmup: int = 2) -> float:
    import torch

    for _ in range(warmup):
        fn()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / reps


def _lengths(default: int, n: int) -> list[int]:
    out = []
    for f in (0.5, 1.0, 2.0):
        v = max(32, min(n, 32 * int(round(default * f / 32))))
        if v not in out:
            out.append(v)
    return out


def tune_solve(S, b, x, stream=None, reps: int = 20) -> dict:
    """Time the one-right-hand-side solve (device tensors b, x) over rows per chain
    in {1/2, 1, 2} x the preprocessing default and stages in {2, 3}; keep the
    fastest.  Returns {"choice": {...}, "ms": {(rows, stages): ms}}."""
    import torch

    stream = stream or torch.cuda.current_stream()
    sp = stream.cuda_stream
    if S.scalar("chain") != 1:
        return {"choice": None, "ms": {}}
    table = {}
    for rows in _lengths(S.scalar("rows"), S.scalar("n")):
        try:
            S.tune("rows", rows)
        except Exception:
            continue  # no valid plan from this length
        for stages in (2, 3):
            S.tune("stages", stages)
            ms = _events_ms(lambda: S.solve_device(b.data_ptr(), x.data_ptr(), sp), stream, reps)
            table[(S.scalar("rows"), stages)] = ms
    (rows, stages) = min(table, key=table.get)
    S.tune("rows", rows).tune("stages", stages)
    return {"choice": {"rows": rows, "stages": stages}, "ms": table}


def tune_batch(S, B, X, mode: int = 0, iters: int = 1, stream=None, reps: int = 5) -> dict:
    """Time batched solves of device tensors B, X (rows = right-hand sides) in
    `mode` with `iters` refinement steps over the path (chain kernels, partition
    kernels) and, on the chain path, the batched plan's rows per task in {1/2, 1,
    2} x its default; keep the fastest.  Returns {"choice": {...}, "ms": {...}}."""
    import torch

    stream = stream or torch.cuda.current_stream()
    sp = stream.cuda_stream
    if S.scalar("chain") != 1:
        return {"choice": None, "ms": {}}

    def run():
        S.solve_batch(B, X, mode=mode, tol=-1.0, maxit=iters, stream=sp, want_resid=False)

    table = {}
    default_rows = S.scalar("batch_rows")
    for rows in _lengths(default_rows, S.scalar("n")):
        try:
            S.tune("batch_rows", rows)
        except Exception:
            continue
        S.tune("batch_path", 1)
        table[("chain", S.scalar("batch_rows"))] = _events_ms(run, stream, reps)
    if not S.scalar("lean"):
        S.tune("batch_path", 0)
        table[("partition", 0)] = _events_ms(run, stream, reps)
    path, rows = min(table, key=table.get)
    if path == "chain":
        S.tune("batch_rows", rows).tune("batch_path", 1)
    else:
        S.tune("batch_rows", default_rows).tune("batch_path", 0)
    return {"choice": {"path": path, "batch_rows": rows or None}, "ms": table}
