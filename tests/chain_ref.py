"""CPU restatement of the chain solve's plan and phases (test infrastructure).

Follows spike_pstrsv_b200/csrc/chain.cu: chains of `length` rows over U (the
working upper-triangular matrix), each chain's spike computed exactly (sparse
triangular solves on the chain's block with the coupling columns as right-hand
sides), f = the first row from the top whose absolute spike-row sum exceeds
tau; phase 1 solves a chain with zero coupling and keeps rows [a, f); phase 4
re-solves rows [f, q) with the values below the chain.  Used by the CPU tests of
the sharded solve (gloo ranks) as the per-rank backend."""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as sla

TAU = 2.0 ** -60


def upper(A, uplo: str):
    """U (the matrix the chains run on) and whether x is reversed."""
    from spike_pstrsv_b200 import synth

    U = A if uplo.upper() == "U" else synth.mirror(A)
    return sp.csr_matrix((U.a, U.ja, U.ia), shape=(U.m, U.m)), uplo.upper() == "L"


def chain_plan(U: sp.csr_matrix, length: int, tau: float = TAU):
    """Phase-1 tasks (lo, hi, st_lo, st_hi) and the column reach of U."""
    n = U.shape[0]
    coo = U.tocoo()
    reach = int((coo.col - coo.row).max())
    tasks = []
    for a in range(0, n, length):
        q = min(a + length, n)
        R = U[a:q, q:]
        f = q
        if R.nnz:
            cols = np.unique(R.nonzero()[1])
            S = sla.spsolve_triangular(U[a:q, a:q].tocsr(), R[:, cols].toarray(), lower=False)
            bad = np.nonzero(~(np.abs(S).sum(axis=1) <= tau))[0]
            if len(bad):
                f = a + int(bad.min())
        tasks.append((a, q, a, f))
    return np.array(tasks, dtype=np.int64).reshape(-1), reach


class NumpyBackend:
    """Both phases of a shard's chains on the CPU (x and b are caller-order torch
    CPU tensors, as the sharded driver passes them)."""

    def __init__(self, U: sp.csr_matrix, rev: bool, tasks1):
        self.U, self.rev = U, rev
        self.t = np.asarray(tasks1).reshape(-1, 4)
        self.n = U.shape[0]

    def _u(self, v):
        v = v.numpy()
        return v[::-1] if self.rev else v

    def phase(self, ph: int, lo: int, hi: int, b, x) -> None:
        bu, xu = self._u(b), self._u(x)  # views (reversed for 'L'), writes land in x
        for a, q, _, f in self.t:
            if ph == 1 and lo <= a and q <= hi:
                y = sla.spsolve_triangular(self.U[a:q, a:q].tocsr(), bu[a:q].copy(), lower=False)
                xu[a:f] = y[: f - a]
            if ph == 4 and f < q and lo < q <= hi:
                rhs = bu[f:q] - self.U[f:q, q:] @ xu[q:]
                xu[f:q] = sla.spsolve_triangular(self.U[f:q, f:q].tocsr(), rhs, lower=False)
