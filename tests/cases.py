"""Small seeded test matrices (upper and lower triangular CSR)."""
from __future__ import annotations

import numpy as np

from spike_pstrsv_b200 import synth


def rand_upper(m: int, dens: float, band: int, far_prob: float, seed: int,
               iso_blocks=None, P: int | None = None) -> synth.CSR:
    """Random upper-triangular CSR, diagonal first: a Binomial(band, dens) count of
    columns within `band` of the diagonal, an occasional far column, optional blocks
    (of an equal P-split) that couple to nothing and are referenced by nothing."""
    rng = np.random.default_rng(seed)
    ia = [0]
    ja: list[int] = []
    a: list[float] = []
    k = m // P if P else 0
    for i in range(m):
        cols = set()
        hi = min(m - 1, i + band)
        if hi > i:
            cnt = rng.binomial(hi - i, dens)
            cols.update((i + 1 + rng.choice(hi - i, size=cnt, replace=False)).tolist())
        if i < m - 1 and rng.random() < far_prob:
            cols.add(int(rng.integers(i + 1, m)))
        if iso_blocks is not None:
            t = min(i // k, P - 1)
            if t in iso_blocks:
                pe = (t + 1) * k if t < P - 1 else m
                cols = {c for c in cols if c < pe}
            cols = {c for c in cols if min(c // k, P - 1) not in iso_blocks or min(c // k, P - 1) == t}
        cols = sorted(cols)
        offs = rng.standard_normal(len(cols)) / 8
        ja += [i] + cols
        a += [1 + float(np.abs(offs).sum())] + offs.tolist()
        ia.append(len(ja))
    return synth.CSR(m, np.array(ia, np.int32), np.array(ja, np.int32), np.array(a))


def random_cases(count: int = 40, base_seed: int = 1000):
    """(name, CSR, P) tuples covering bands, far couplings and isolated blocks."""
    out = []
    for seed in range(count):
        rng = np.random.default_rng(base_seed + seed)
        m = int(rng.integers(20, 400))
        P = int(rng.integers(1, min(m, 24) + 1))
        band = int(rng.integers(1, 40))
        dens = float(rng.uniform(0.05, 0.9))
        far = float(rng.choice([0.0, 0.01, 0.1]))
        iso = None
        if seed % 3 == 0 and P >= 3:
            iso = set(rng.choice(P, size=max(1, P // 3), replace=False).tolist())
        out.append((f"rand{seed}", rand_upper(m, dens, band, far, seed, iso, P), P))
    return out


def rel_err(x, y) -> float:
    return float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-300))


def struct_diff(got: dict, want: dict) -> list:
    """Names of structure entries that are not bit-identical."""
    bad = []
    for k, w in want.items():
        g = got[k]
        if isinstance(w, np.ndarray):
            g = np.asarray(g)
            if g.shape != w.shape or g.dtype.itemsize != w.dtype.itemsize:
                bad.append(k)
            elif w.dtype == np.float64:
                if not np.array_equal(g.view(np.uint64), w.view(np.uint64)):
                    bad.append(k)
            elif not np.array_equal(g.astype(np.int64), w.astype(np.int64)):
                bad.append(k)
        elif int(g) != int(w):
            bad.append(k)
    return bad
