"""Test checker: a plain-Python restatement of the reordering's partitioner
(reverse Cuthill-McKee from a George-Liu pseudo-peripheral node per component,
searched from the component's lightest node,
neighbours by increasing degree then index, cut into ranges of nearly equal row
nonzeros) and of the reference's later steps (src/matrix_reordering.c:152-264:
rows grouped by partition in original order, the permuted matrix's triangle as
CSR with sorted columns).  Small inputs only."""
from __future__ import annotations

import numpy as np


def sym_pattern(n, ia, ja):
    rows = [set() for _ in range(n)]
    for r in range(n):
        for k in range(ia[r], ia[r + 1]):
            c = int(ja[k])
            if c != r:
                rows[r].add(c)
                rows[c].add(r)
    return [sorted(s) for s in rows]


def _levels(adj, root):
    seen = {root}
    levels = [[root]]
    while True:
        nxt = []
        for v in levels[-1]:
            for u in adj[v]:
                if u not in seen:
                    seen.add(u)
                    nxt.append(u)
        if not nxt:
            return levels
        levels.append(nxt)


def rcm_order(n, ia, ja):
    adj = sym_pattern(n, ia, ja)
    key = lambda v: (len(adj[v]), v)  # noqa: E731
    order, placed = [], [False] * n
    for s0 in range(n):
        if placed[s0]:
            continue
        if not adj[s0]:
            root = s0
        else:
            lv = _levels(adj, s0)
            root = min((v for l in lv for v in l), key=key)
            if root != s0:
                lv = _levels(adj, root)
            for _ in range(32):
                x = min(lv[-1], key=key)
                lx = _levels(adj, x)
                if len(lx) <= len(lv):
                    break
                root, lv = x, lx
        head = len(order)
        order.append(root)
        placed[root] = True
        while head < len(order):
            v = order[head]
            head += 1
            new = [u for u in adj[v] if not placed[u]]
            for u in new:
                placed[u] = True
            order.extend(sorted(new, key=key))
    return np.array(order[::-1], dtype=np.int32)


def cut(n, ia, order, nparts):
    w = np.maximum(1, np.diff(np.asarray(ia, dtype=np.int64)))
    total = int(w.sum())
    bound = [0] * (nparts + 1)
    bound[nparts] = n
    acc, q = 0, 0
    for k in range(1, nparts):
        while q < n and acc * nparts < total * k:
            acc += int(w[order[q]])
            q += 1
        bound[k] = min(max(q, bound[k - 1] + 1), n - (nparts - k))
    part = np.zeros(n, dtype=np.int32)
    for k in range(nparts):
        part[order[bound[k]:bound[k + 1]]] = k
    return part


def plan(n, ia, ja, nparts):
    order = rcm_order(n, ia, ja)
    return order, cut(n, ia, order, nparts)


def grouped_perm(part, nparts):
    """Rows grouped by partition, original order inside (src/matrix_reordering.c:152-172)."""
    perm = np.concatenate([np.flatnonzero(part == t) for t in range(nparts)]).astype(np.int32)
    sizes = np.bincount(part, minlength=nparts).astype(np.int32)
    return perm, sizes


def permuted_triangle(A_csr, perm, uplo):
    """Triangle of P A P^T (row i = row perm[i]) as sorted CSR (a, ia, ja)."""
    import scipy.sparse as sp

    n = A_csr.shape[0]
    iperm = np.empty(n, dtype=np.int64)
    iperm[perm] = np.arange(n)
    C = A_csr.tocoo()
    r, c = iperm[C.row], iperm[C.col]
    keep = c >= r if uplo.upper() == "U" else c <= r
    B = sp.csr_matrix((C.data[keep], (r[keep], c[keep])), shape=(n, n))
    B.sort_indices()
    return B.data, B.indptr.astype(np.int32), B.indices.astype(np.int32)
