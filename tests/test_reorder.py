"""Partition-aware reordering: the host partitioner (spk_reorder_plan, no GPU)
against the plain-Python restatement in reorder_ref.py, and its bandwidth against
scipy's reverse Cuthill-McKee."""
import numpy as np
import pytest
import scipy.sparse as sp
from scipy.sparse.csgraph import reverse_cuthill_mckee

import spike_pstrsv_b200 as spk
from reorder_ref import plan as ref_plan


def scrambled(A, seed):
    n = A.shape[0]
    p = np.random.default_rng(seed).permutation(n)
    B = (sp.csr_matrix(A)[p][:, p] + sp.eye(n)).tocsr()
    B.sort_indices()
    return B


def grid(k):
    T = sp.diags([-1.0, 4.0, -1.0], [-1, 0, 1], (k, k))
    return (sp.kron(sp.eye(k), T) + sp.kron(sp.diags([-1.0, -1.0], [-1, 1], (k, k)), sp.eye(k))).tocsr()


def random_sym(n, dens, seed):
    R = sp.random(n, n, density=dens, random_state=seed, format="csr")
    return (R + R.T).tocsr()


def bandwidth(A, order):
    n = A.shape[0]
    pos = np.empty(n, dtype=np.int64)
    pos[order] = np.arange(n)
    C = A.tocoo()
    return int(np.max(np.abs(pos[C.row] - pos[C.col]))) if C.nnz else 0


CASES = {
    "grid24": lambda: scrambled(grid(24), 1),
    "band7": lambda: scrambled(sp.diags([1.0] * 15, list(range(-7, 8)), (700, 700)), 2),
    "rand_components": lambda: scrambled(sp.block_diag([random_sym(150, 0.03, 3), random_sym(90, 0.05, 4),
                                                        sp.eye(20)]), 5),
    "unsymmetric": lambda: (sp.random(300, 300, density=0.01, random_state=6, format="csr") + sp.eye(300)).tocsr(),
}


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("P", [1, 4, 13])
def test_plan_matches_restatement(name, P):
    A = CASES[name]()
    A.sort_indices()
    n = A.shape[0]
    order, part = spk.reorder_plan(A.indptr, A.indices, n, P)
    o_ref, p_ref = ref_plan(n, A.indptr, A.indices, P)
    assert np.array_equal(order, o_ref)
    assert np.array_equal(part, p_ref)
    assert np.array_equal(np.sort(order), np.arange(n))
    sizes = np.bincount(part, minlength=P)
    assert (sizes > 0).all() and sizes.sum() == n
    # every partition is a contiguous range of the order
    pos = np.empty(n, dtype=np.int64)
    pos[order] = np.arange(n)
    for t in range(P):
        q = np.sort(pos[part == t])
        assert q[-1] - q[0] + 1 == len(q)


@pytest.mark.parametrize("name", ["grid24", "band7", "rand_components"])
def test_bandwidth_as_scipy_rcm(name):
    A = CASES[name]()
    order, _ = spk.reorder_plan(A.indptr, A.indices, A.shape[0], 2)
    ours = bandwidth(A, order)
    theirs = bandwidth(A, reverse_cuthill_mckee(A, symmetric_mode=True))
    assert ours <= max(theirs + 2, int(1.1 * theirs)), (ours, theirs)
    if name != "rand_components":  # random graphs are expanders: no order makes them narrow
        assert ours < bandwidth(A, np.arange(A.shape[0])) // 4


def test_balanced_by_nonzeros():
    A = scrambled(sp.diags([1.0] * 9, list(range(-4, 5)), (4000, 4000)), 7)
    _, part = spk.reorder_plan(A.indptr, A.indices, A.shape[0], 8)
    w = np.diff(A.indptr)
    loads = np.array([w[part == t].sum() for t in range(8)])
    assert loads.max() <= loads.mean() * 1.01 + 9


def test_plan_rejects_bad_input():
    A = grid(4)
    with pytest.raises(spk.SpkError):
        spk.reorder_plan(A.indptr, A.indices, 16, 17)  # more partitions than rows
    bad = A.indices.copy()
    bad[3] = 99
    with pytest.raises(spk.SpkError):
        spk.reorder_plan(A.indptr, bad, 16, 2)


class Csr:
    """(a, ia, ja, m) of a scipy matrix, the shape the checker wrappers take."""

    def __init__(self, A):
        A = sp.csr_matrix(A)
        A.sort_indices()
        self.a = A.data.astype(np.float64)
        self.ia = A.indptr.astype(np.int32)
        self.ja = A.indices.astype(np.int32)
        self.m = A.shape[0]


@pytest.mark.skipif(not __import__("oracle").Reference.available(),
                    reason=__import__("oracle").Reference.missing_reason())
@pytest.mark.parametrize("uplo", ["U", "L"])
def test_restatement_pinned_to_reference_steps(uplo):
    """The reference's matrixReordering, its METIS call answered with a given
    partition, against grouped_perm + permuted_triangle (the checker the GPU
    tests use)."""
    import oracle
    from reorder_ref import grouped_perm, permuted_triangle

    A = scrambled(grid(20), 9)
    F = Csr(A)
    P = 5
    part = np.random.default_rng(3).integers(0, P, F.m).astype(np.int32)
    part[:P] = np.arange(P)
    R = oracle.Reference()
    ra, ria, rja, starts, ends, nrows = R.reorder(F, P, uplo, part)
    R.set_flag("IS_MATRIX_PARTITIONED", 0)
    perm, sizes = grouped_perm(part, P)
    a, ia, ja = permuted_triangle(A, perm, uplo)
    assert np.array_equal(ria, ia) and np.array_equal(rja, ja)
    assert np.array_equal(ra.view(np.uint64), a.view(np.uint64))
    assert np.array_equal(nrows, sizes)
    assert np.array_equal(starts, np.concatenate([[0], np.cumsum(sizes)[:-1]]))
    assert np.array_equal(ends, np.cumsum(sizes))


@pytest.mark.skipif(not __import__("oracle").Reference.available(),
                    reason=__import__("oracle").Reference.missing_reason())
def test_oracle_lower_caller_partitions_pinned_to_reference():
    """Caller partitions of an 'L' matrix are in L's row order; the oracle maps
    partition t to partition P-1-t of the mirror J L J.  The reference (which runs
    'U' only) given the mirrored bounds builds the same structure."""
    import oracle
    from spike_pstrsv_b200 import synth
    from test_oracle_pins import trim_S
    from cases import struct_diff

    L = synth.poisson2d_lower(32)
    n, P = L.m, 5
    sizes = np.array([200, 180, 250, 190, n - 820])
    ends = np.cumsum(sizes)
    starts = ends - sizes
    R = oracle.Reference()
    R.set_partitions(n - ends[::-1], n - starts[::-1])
    R.preproc(synth.mirror(L), P)
    want = R.structure()
    O = oracle.Oracle()
    assert O.preproc(L, P, uplo="L", flb=1, starts=starts, ends=ends) == 0
    assert list(O.array("partition_starts")) == list(n - ends[::-1])
    assert struct_diff(trim_S(O.structure(), len(want["S"])), want) == []
