"""Partition-aware reordering on the GPU (matrixReordering / spk_reorder, the
role of src/matrix_reordering.c:83-305) against the reference's own reordering
steps (oracle/_ref: its matrixReordering given the RCM-ordered matrix, its METIS
call answered with the same contiguous partitions) and the checker restatement;
then the Spike preprocessing and solve of the reordered triangle with the
reordering's partitions (IS_MATRIX_PARTITIONED) against the reference's.
Structure bit-identical, x to relative error <= 1e-12."""
import numpy as np
import pytest

import oracle
import spike_pstrsv_b200 as spk
from cases import rel_err, struct_diff
from reorder_ref import grouped_perm, permuted_triangle
from test_oracle_pins import trim_S
from test_reorder import CASES, Csr, grid, scrambled

pytestmark = pytest.mark.gpu
TOL = 1e-12
needs_ref = pytest.mark.skipif(not oracle.Reference.available(), reason=oracle.Reference.missing_reason())


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("uplo", ["U", "L"])
def test_reorder_matches_restatement(name, uplo):
    A = CASES[name]()
    F = Csr(A)
    P = 6
    a, ia, ja, perm = spk.reorder(F.a, F.ia, F.ja, F.m, P, uplo)
    order, part = spk.reorder_plan(F.ia, F.ja, F.m, P)  # the host-built graph gives the same plan
    assert np.array_equal(perm, order)
    perm_ref, sizes = grouped_perm(part[order], P)  # parts are ranges of the order: grouping keeps it
    assert np.array_equal(perm_ref, np.arange(F.m))
    assert [spk.get_global("partition_numRows", t) for t in range(P)] == list(sizes)
    ra, ria, rja = permuted_triangle(A, order, uplo)
    assert np.array_equal(ia, ria) and np.array_equal(ja, rja)
    assert np.array_equal(a.view(np.uint64), ra.view(np.uint64))
    assert spk.get_flag("IS_MATRIX_PARTITIONED") == 1
    spk.set_flag("IS_MATRIX_PARTITIONED", 0)


@needs_ref
@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("P", [3, 8])
def test_matrix_reordering_matches_reference(uplo, P):
    A = scrambled(grid(40), 11)
    F = Csr(A)
    order, part = spk.reorder_plan(F.ia, F.ja, F.m, P)
    R = oracle.Reference()
    # the reference's steps on the RCM-ordered matrix with the same (contiguous) parts
    ra, ria, rja, rs, re, rn = R.reorder(Csr(A[order][:, order]), P, uplo, part[order])
    R.set_flag("IS_MATRIX_PARTITIONED", 0)
    a, ia, ja, _ = spk.reorder(F.a, F.ia, F.ja, F.m, P, uplo, legacy=True)
    assert spk.get_flag("IS_MATRIX_PARTITIONED") == 1
    spk.set_flag("IS_MATRIX_PARTITIONED", 0)
    assert np.array_equal(ia, ria) and np.array_equal(ja, rja)
    assert np.array_equal(a.view(np.uint64), ra.view(np.uint64))
    for name, want in (("partition_starts", rs), ("partition_ends", re), ("partition_numRows", rn)):
        assert [spk.get_global(name, t) for t in range(P)] == list(want), name


@needs_ref
@pytest.mark.parametrize("P", [4, 12])
def test_reordered_system_solves_as_reference(P):
    """matrixReordering -> spike_pstrsv_preproc (caller partitions) -> solve, as the
    reference's profiler drives it with METIS (test/runtime_analysis.c:297-310, 413-427)."""
    A = scrambled(grid(48), 12)
    F = Csr(A)
    order, part = spk.reorder_plan(F.ia, F.ja, F.m, P)
    R = oracle.Reference()
    ra, ria, rja, *_ = R.reorder(Csr(A[order][:, order]), P, "U", part[order])

    class U:
        a, ia, ja, m = ra, ria, rja, F.m

    R.preproc(U, P)  # consumes the reference's IS_MATRIX_PARTITIONED
    a, ia, ja, _ = spk.reorder(F.a, F.ia, F.ja, F.m, P, "U", legacy=True)
    import scipy.sparse as sp

    M = sp.csr_matrix((a, ja, ia), shape=(F.m, F.m))
    x_true = np.random.default_rng(0).uniform(-1, 1, F.m)
    b = M @ x_true
    x = np.zeros(F.m)
    spk.spike_pstrsv_preproc(a, ia, ja, F.m, P, "U")
    assert spk.get_flag("IS_MATRIX_PARTITIONED") == 0
    spk.spike_pstrsv_solve("U", F.m, b.copy(), x, P)
    want = R.structure()
    got = trim_S(spk.legacy_structure(), len(want["S"]))
    assert struct_diff(got, want) == []
    assert rel_err(x, R.solve(b)) <= TOL
    assert rel_err(x, x_true) <= TOL
    # the reordering leaves a block coupled only to the next one
    starts = [spk.get_global("partition_starts", t) for t in range(P)]
    ends = [spk.get_global("partition_ends", t) for t in range(P)]
    for t in range(P - 1):
        cols = ja[ia[starts[t]]:ia[ends[t]]]
        assert cols.max() < ends[t + 1]


def test_analysis_keeps_decoupled_matrix():
    """Equal partitions that already decouple: matrixAnalysis returns 1 and the
    matrix becomes its triangle, nothing reordered (src/matrix_reordering.c:307-356)."""
    import scipy.sparse as sp

    blocks = [grid(8) for _ in range(4)]
    A = sp.block_diag(blocks).tocsr()
    F = Csr(A)
    a, ia, ja, _ = spk.reorder(F.a, F.ia, F.ja, F.m, 4, "U", legacy=True)
    T = sp.triu(A).tocsr()
    T.sort_indices()
    assert np.array_equal(ia, T.indptr) and np.array_equal(ja, T.indices)
    assert np.array_equal(a, T.data)
    assert spk.get_flag("IS_MATRIX_PARTITIONED") == 0


@pytest.mark.parametrize("P", [3, 9])
def test_reordered_lower_system_matches_oracle(P):
    """matrixReordering with uplo 'L' -> spike_pstrsv_preproc 'L' with the
    reordering's partitions (in L's row order, mirrored for the J L J structure)
    -> solve, against the oracle given the same partitions."""
    A = scrambled(grid(40), 13)
    F = Csr(A)
    a, ia, ja, _ = spk.reorder(F.a, F.ia, F.ja, F.m, P, "L", legacy=True)
    n = F.m
    starts = np.array([spk.get_global("partition_starts", t) for t in range(P)])
    ends = np.array([spk.get_global("partition_ends", t) for t in range(P)])

    class Lm:
        pass

    Lm.a, Lm.ia, Lm.ja, Lm.m = a, ia, ja, n
    O = oracle.Oracle()
    assert O.preproc(Lm, P, uplo="L", flb=1, starts=starts, ends=ends) == 0
    import scipy.sparse as sp

    x_true = np.random.default_rng(1).uniform(-1, 1, n)
    b = sp.csr_matrix((a, ja, ia), shape=(n, n)) @ x_true
    x = np.zeros(n)
    spk.spike_pstrsv_preproc(a, ia, ja, n, P, "L")
    assert spk.get_flag("IS_MATRIX_PARTITIONED") == 0
    spk.spike_pstrsv_solve("L", n, b.copy(), x, P)
    st = spk.legacy_structure()
    assert list(st["partition_starts"]) == list(n - ends[::-1])
    assert struct_diff(st, O.structure()) == []
    assert rel_err(x, O.solve(b)) <= TOL
    assert rel_err(x, x_true) <= TOL
    # each block of L couples only to the block before it
    for t in range(1, P):
        cols = ja[ia[starts[t]]:ia[ends[t]]]
        assert cols.min() >= starts[t - 1]
