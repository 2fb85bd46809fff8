"""Seeded synthetic CSR matrices with the shapes of the spike_pstrsv workloads.

The reference runs on external MatrixMarket files (test/runtime_analysis.c:279-292,
tools/autoExperiments.sh:2-8) that are not available; these generators stand in
for them.  All matrices are 0-based CSR with int32 ``ia``/``ja``, float64 values,
sorted column indices and the diagonal present (last entry of a lower-triangular
row, first entry of an upper-triangular row), which is the input contract of the
reference's solver (spike_pstrsv_ops.c:1179-1194 reads the diagonal as the first
entry of an upper row).

Random numbers come from numpy's PCG64 (``numpy.random.default_rng(seed)``).

Workloads:
  * ``poisson2d_lower(128)``   lower triangle of the 5-point Poisson matrix on a
    128x128 grid: m = 16,384, nnz = 48,896, diagonal 4, off-diagonals -1.
  * ``banded_lower(4194304)``  each row i has min(i, 16) off-diagonals at distinct
    columns drawn uniformly from [max(0, i-64), i-1]; values N(0,1)/16, diagonal
    1 + sum|off|: m = 4,194,304, nnz = 17m - 136 = 71,303,032.
  * ``ic0_laplace3d_lower(128)`` IC(0)-style factor of the 7-point Laplacian on a
    128^3 grid: diagonal sqrt(6), off-diagonals -1/sqrt(6) x U(0.9, 1.1):
    m = 2,097,152, nnz = 8,339,456.
  * ``poisson_banded_lower``   off-diagonals per row ~ Poisson(mean) inside a band
    (the batched and serving pools).
"""
from __future__ import annotations

import dataclasses

import numpy as np

__all__ = [
    "CSR",
    "poisson2d_lower",
    "banded_lower",
    "ic0_laplace3d_lower",
    "poisson_banded_lower",
    "transpose",
    "mirror",
    "spmv",
    "make_rhs",
    "batch_pool",
]


@dataclasses.dataclass
class CSR:
    """0-based CSR matrix (int32 indices, float64 values)."""

    m: int
    ia: np.ndarray
    ja: np.ndarray
    a: np.ndarray

    @property
    def nnz(self) -> int:
        return int(self.ia[-1])

    def astuple(self):
        return self.m, self.ia, self.ja, self.a


def _csr_from_rows(m, row_len, cols, vals):
    ia = np.zeros(m + 1, dtype=np.int64)
    np.cumsum(row_len, out=ia[1:])
    return CSR(m, ia.astype(np.int32), cols.astype(np.int32), vals.astype(np.float64))


def poisson2d_lower(n: int = 128) -> CSR:
    """Lower triangle (with diagonal) of the 5-point Poisson matrix on an n x n grid."""
    m = n * n
    i = np.arange(m, dtype=np.int64)
    gx = i % n
    gy = i // n
    has_s = gy > 0
    has_w = gx > 0
    row_len = 1 + has_s.astype(np.int64) + has_w.astype(np.int64)
    ia = np.zeros(m + 1, dtype=np.int64)
    np.cumsum(row_len, out=ia[1:])
    nnz = int(ia[-1])
    ja = np.empty(nnz, dtype=np.int64)
    a = np.empty(nnz, dtype=np.float64)
    pos = ia[:-1].copy()
    ja[pos[has_s]] = i[has_s] - n
    a[pos[has_s]] = -1.0
    pos[has_s] += 1
    ja[pos[has_w]] = i[has_w] - 1
    a[pos[has_w]] = -1.0
    pos[has_w] += 1
    ja[pos] = i
    a[pos] = 4.0
    return CSR(m, ia.astype(np.int32), ja.astype(np.int32), a)


def banded_lower(m: int = 4194304, per_row: int = 16, band: int = 64, seed: int = 0,
                 chunk: int = 1 << 18) -> CSR:
    """Row i: min(i, per_row) distinct columns uniform in [max(0, i-band), i-1] plus the
    diagonal.  Off-diagonal values N(0,1)/16, diagonal 1 + sum of |off-diagonals|."""
    rng = np.random.default_rng(seed)
    row_len = np.minimum(np.arange(m, dtype=np.int64), per_row) + 1
    ia = np.zeros(m + 1, dtype=np.int64)
    np.cumsum(row_len, out=ia[1:])
    nnz = int(ia[-1])
    ja = np.empty(nnz, dtype=np.int32)
    a = np.empty(nnz, dtype=np.float64)
    for r0 in range(0, m, chunk):
        r1 = min(m, r0 + chunk)
        rows = np.arange(r0, r1, dtype=np.int64)
        nr = r1 - r0
        # offsets d in [1, band]: column = i - d; keys pick per_row smallest among valid d
        keys = rng.random((nr, band), dtype=np.float32)
        d = np.arange(1, band + 1, dtype=np.int64)
        keys[d[None, :] > rows[:, None]] = np.inf
        k = min(per_row, band)
        pick = np.argpartition(keys, k - 1, axis=1)[:, :k] + 1  # chosen offsets
        cols = rows[:, None] - pick
        valid = np.take_along_axis(keys, pick - 1, axis=1) != np.inf
        cols = np.where(valid, cols, np.int64(1) << 40)
        cols.sort(axis=1)
        nvalid = valid.sum(axis=1)
        offv = rng.standard_normal((nr, k)) / 16.0
        offv = np.where(np.arange(k)[None, :] < nvalid[:, None], offv, 0.0)
        diag = 1.0 + np.abs(offv).sum(axis=1)
        # scatter: each row = its valid sorted cols, then the diagonal
        base = ia[r0:r1]
        mask = np.arange(k)[None, :] < nvalid[:, None]
        dst = base[:, None] + np.arange(k)[None, :]
        ja[dst[mask]] = cols[mask]
        a[dst[mask]] = offv[mask]
        ja[base + nvalid] = rows
        a[base + nvalid] = diag
    return CSR(m, ia.astype(np.int32), ja, a)


def ic0_laplace3d_lower(n: int = 128, seed: int = 0) -> CSR:
    """IC(0)-style lower factor of the 7-point Laplacian on an n^3 grid."""
    rng = np.random.default_rng(seed)
    m = n * n * n
    i = np.arange(m, dtype=np.int64)
    gx = i % n
    gy = (i // n) % n
    gz = i // (n * n)
    nb = [(gz > 0, n * n), (gy > 0, n), (gx > 0, 1)]  # ascending column order
    row_len = 1 + sum(h.astype(np.int64) for h, _ in nb)
    ia = np.zeros(m + 1, dtype=np.int64)
    np.cumsum(row_len, out=ia[1:])
    nnz = int(ia[-1])
    ja = np.empty(nnz, dtype=np.int64)
    a = np.empty(nnz, dtype=np.float64)
    pos = ia[:-1].copy()
    off = -1.0 / np.sqrt(6.0)
    for has, step in nb:
        ja[pos[has]] = i[has] - step
        pos[has] += 1
    ja[pos] = i
    a[:] = off * rng.uniform(0.9, 1.1, size=nnz)
    a[pos] = np.sqrt(6.0)
    return CSR(m, ia.astype(np.int32), ja.astype(np.int32), a)


def poisson_banded_lower(m: int, mean: float, band: int, seed: int) -> CSR:
    """Row i: min(Poisson(mean), i, band) distinct columns uniform in [max(0,i-band), i-1];
    values as in ``banded_lower`` (N(0,1)/16, diagonal 1 + sum|off|)."""
    rng = np.random.default_rng(seed)
    rows = np.arange(m, dtype=np.int64)
    cnt = np.minimum(np.minimum(rng.poisson(mean, size=m), rows), band).astype(np.int64)
    kmax = int(cnt.max()) if m else 0
    keys = rng.random((m, band), dtype=np.float32)
    d = np.arange(1, band + 1, dtype=np.int64)
    keys[d[None, :] > rows[:, None]] = np.inf
    order = np.argsort(keys, axis=1)[:, :max(kmax, 1)] + 1
    take = np.arange(max(kmax, 1))[None, :] < cnt[:, None]
    cols = np.where(take, rows[:, None] - order, np.int64(1) << 40)
    cols.sort(axis=1)
    offv = np.where(take, rng.standard_normal(cols.shape) / 16.0, 0.0)
    diag = 1.0 + np.abs(offv).sum(axis=1)
    row_len = cnt + 1
    ia = np.zeros(m + 1, dtype=np.int64)
    np.cumsum(row_len, out=ia[1:])
    nnz = int(ia[-1])
    ja = np.empty(nnz, dtype=np.int32)
    a = np.empty(nnz, dtype=np.float64)
    base = ia[:-1]
    dst = base[:, None] + np.arange(cols.shape[1])[None, :]
    ja[dst[take]] = cols[take]
    a[dst[take]] = offv[take]
    ja[base + cnt] = rows
    a[base + cnt] = diag
    return CSR(m, ia.astype(np.int32), ja, a)


def transpose(A: CSR) -> CSR:
    """CSR of A^T with sorted column indices (U = L^T keeps the diagonal first)."""
    m, nnz = A.m, A.nnz
    rows = np.repeat(np.arange(m, dtype=np.int64), np.diff(A.ia.astype(np.int64)))
    order = np.lexsort((rows, A.ja))
    cnt = np.bincount(A.ja, minlength=m)
    ia = np.zeros(m + 1, dtype=np.int64)
    np.cumsum(cnt, out=ia[1:])
    return CSR(m, ia.astype(np.int32), rows[order].astype(np.int32), A.a[order].copy())


def mirror(A: CSR) -> CSR:
    """J A J with J the index reversal i -> m-1-i.  A lower-triangular A becomes
    upper triangular with the diagonal first; row r of the result is row m-1-r of A
    reversed, with column c mapped to m-1-c."""
    m, nnz = A.m, A.nnz
    ia = (nnz - A.ia[::-1]).astype(np.int32)
    ja = (m - 1 - A.ja[::-1]).astype(np.int32)
    return CSR(m, ia, ja, A.a[::-1].copy())


def spmv(A: CSR, x: np.ndarray) -> np.ndarray:
    """y = A x in float64, summed in CSR order per row (numpy reduceat)."""
    prod = A.a * x[A.ja]
    y = np.add.reduceat(prod, A.ia[:-1].astype(np.int64)) if A.nnz else np.zeros(A.m)
    y[np.diff(A.ia) == 0] = 0.0
    return y


def make_rhs(A: CSR, seed: int = 0, nrhs: int | None = None):
    """x_true ~ U(-1,1) (seeded), b = A x_true.  Returns (x_true, b)."""
    rng = np.random.default_rng(seed)
    if nrhs is None:
        x = rng.uniform(-1.0, 1.0, size=A.m)
        return x, spmv(A, x)
    X = rng.uniform(-1.0, 1.0, size=(nrhs, A.m))
    return X, np.stack([spmv(A, X[k]) for k in range(nrhs)])


def batch_pool(count: int = 512, m_lo: int = 1024, m_hi: int = 262144, band_lo: int = 32,
               band_hi: int = 256, mean: float = 8.0, seed: int = 0,
               rhs_choices=(1, 2, 4, 8, 16, 32)):
    """Systems of the batched workload: m log-uniform in [m_lo, m_hi], off-diagonals per
    row ~ Poisson(mean) within a per-system band in [band_lo, band_hi], k right-hand
    sides drawn from ``rhs_choices``.  Returns a list of (CSR, nrhs)."""
    rng = np.random.default_rng(seed)
    ms = np.exp(rng.uniform(np.log(m_lo), np.log(m_hi), size=count)).astype(np.int64)
    bands = rng.integers(band_lo, band_hi + 1, size=count)
    ks = rng.choice(np.asarray(rhs_choices), size=count)
    seeds = rng.integers(0, 2**31 - 1, size=count)
    return [(poisson_banded_lower(int(ms[i]), mean, int(bands[i]), int(seeds[i])), int(ks[i]))
            for i in range(count)]
