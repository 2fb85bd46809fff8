"""A chain solve whose rows are sharded over the ranks of a torch.distributed
group, one GPU per rank.

The reference solves one system with one OpenMP team; its only exchange is
the barrier before the reduced system (src/spike_pstrsv.c:201-210).  The chain
solve has the same shape: phase 1 solves every chain with zero coupling,
phase 4 re-solves the coupled rows of each chain from the values at the rows
just below it.  Sharding keeps that order:

* rank r owns the U rows [lo_r, hi_r), a run of whole chains (the plan splits
  the chains into `world` runs of nearly equal row counts);
* phase 1 of its chains runs with no communication;
* exchange: rank r sends x at its first `reach` rows (final after phase 1) to
  rank r-1 and receives the `reach` rows after hi_r from rank r+1 (one
  point-to-point message of reach doubles each way per solve; NCCL send/recv
  over NVLink on GPUs, gloo on CPU);
* phase 4 of its chains runs with those rows in x.

A backend runs the two phases on the rank's device: ``DeviceBackend`` calls the
library's ``spk_chain_phase`` on CUDA tensors.  Buffers are full length (the
caller's order); each rank reads and writes only its rows and the halo.
"""
from __future__ import annotations

import numpy as np


def plan(tasks1: np.ndarray, world: int) -> list[tuple[int, int]]:
    """Row ranges (U order) of `world` shards of whole chains.  tasks1 holds the
    phase-1 tasks as rows (lo, hi, st_lo, st_hi) in row order."""
    t = np.asarray(tasks1).reshape(-1, 4)
    if len(t) < world:
        raise ValueError(f"{len(t)} chains cannot be split over {world} ranks")
    ends = t[:, 1].astype(np.int64)
    n = int(ends[-1])
    cuts = [0]
    for r in range(1, world):
        target = n * r // world
        c = int(np.searchsorted(ends, target))  # first chain ending at or after the target
        c = min(max(c, cuts[-1] + 1), len(t) - (world - r))
        cuts.append(c)
    cuts.append(len(t))
    return [(int(t[cuts[r], 0]), int(t[cuts[r + 1] - 1, 1])) for r in range(world)]


def caller_slice(n: int, rev: bool, a: int, b: int) -> slice:
    """Caller-order indices of U rows [a, b) (uplo 'L': U row r is caller row n-1-r)."""
    a, b = max(0, min(a, n)), max(0, min(b, n))
    return slice(n - b, n - a) if rev else slice(a, b)


def exchange(x, n: int, rev: bool, lo: int, hi: int, reach: int, rank: int, world: int, group=None) -> None:
    """Send x at U rows [lo, lo+reach) to rank-1; receive U rows [hi, hi+reach) from
    rank+1 into x (torch tensors; NCCL on CUDA tensors, gloo on CPU ones)."""
    import torch.distributed as dist

    ops = []
    if rank > 0:
        ops.append(dist.P2POp(dist.isend, x[caller_slice(n, rev, lo, lo + reach)].contiguous(), rank - 1, group))
    if rank + 1 < world and hi < n:
        buf = x[caller_slice(n, rev, hi, hi + reach)]
        ops.append(dist.P2POp(dist.irecv, buf, rank + 1, group))
    if ops:
        for w in dist.batch_isend_irecv(ops):
            w.wait()


class DeviceBackend:
    """The two phases of a rank's chains on its GPU (spk_chain_phase)."""

    def __init__(self, system, stream=None):
        self.system = system
        self.stream = stream

    def phase(self, ph: int, lo: int, hi: int, b, x) -> None:
        import torch

        st = self.stream if self.stream is not None else torch.cuda.current_stream()
        self.system.chain_phase(ph, lo, hi, b.data_ptr(), x.data_ptr(), st.cuda_stream)

    def sync(self) -> None:
        import torch

        (self.stream if self.stream is not None else torch.cuda.current_stream()).synchronize()


class ShardedSolve:
    """One rank's part of a sharded chain solve (see the module docstring)."""

    def __init__(self, backend, n: int, uplo: str, reach: int, tasks1, rank: int, world: int, group=None):
        self.backend = backend
        self.n, self.rev, self.reach = int(n), uplo.upper() == "L", int(reach)
        self.rank, self.world, self.group = rank, world, group
        self.ranges = plan(tasks1, world)
        self.lo, self.hi = self.ranges[rank]

    @classmethod
    def from_system(cls, system, rank: int, world: int, group=None, stream=None):
        if system.scalar("chain") != 1:
            raise ValueError("the system is not solved by chains (exact mode, or rows the chains cannot cover)")
        return cls(DeviceBackend(system, stream), system.n, system.uplo, system.scalar("chain_reach"),
                   system.array("chain_tasks1"), rank, world, group)

    def rows(self) -> slice:
        """This rank's rows of x, caller order."""
        return caller_slice(self.n, self.rev, self.lo, self.hi)

    def solve(self, b, x) -> None:
        """x[rows()] for right-hand side b (full-length buffers; b must hold this
        rank's rows, x receives this rank's rows and its halo)."""
        self.backend.phase(1, self.lo, self.hi, b, x)
        if hasattr(self.backend, "sync"):
            self.backend.sync()  # the halo this rank sends is written by its phase 1
        exchange(x, self.n, self.rev, self.lo, self.hi, self.reach, self.rank, self.world, self.group)
        self.backend.phase(4, self.lo, self.hi, b, x)
