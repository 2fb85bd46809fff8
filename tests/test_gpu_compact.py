"""spk_compact (serving residency): a system solved by chains keeps only what
its solves read.  The compacted system must give the same results as before on
every solve path that remains open (single host / device solves, batched FP64
and FP32 + refinement, which take the chain kernels), hold far fewer device
bytes, refuse the paths that need the released pools, and come back whole when
preprocessed again."""
import numpy as np
import pytest

import oracle
import spike_pstrsv_b200 as spk
from cases import rel_err
from spike_pstrsv_b200 import synth
from spike_pstrsv_b200.capi import SpkError

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.mark.parametrize("uplo", ["L", "U"])
def test_compact_keeps_results_and_frees_pools(monkeypatch, uplo):
    import torch

    monkeypatch.setenv("SPK_CHAIN_BATCH", "1")  # the uncompacted reference takes the same kernels
    L = synth.banded_lower(150001, seed=21)
    A = L if uplo == "L" else synth.transpose(L)
    Xt, B = synth.make_rhs(A, seed=21, nrhs=9)
    S = spk.System().preproc(A.a, A.ia, A.ja, A.m, 37, uplo, 1)
    assert S.scalar("chain") == 1
    x_full = S.solve(B[0])
    dB = torch.from_numpy(B).cuda()
    dX0 = torch.zeros_like(dB)
    S.solve_batch(dB, dX0, mode=0)
    X0 = dX0.cpu().numpy()
    bytes_full = S.scalar("device_bytes")

    freed = S.compact()
    assert S.scalar("lean") == 1
    assert freed > 0 and S.scalar("device_bytes") == bytes_full - freed
    assert S.scalar("device_bytes") < 0.6 * bytes_full
    # same results on the open paths
    assert np.array_equal(S.solve(B[0]), x_full)
    dX = torch.zeros_like(dB)
    S.solve_batch(dB, dX, mode=0)
    assert np.array_equal(dX.cpu().numpy(), X0)
    assert rel_err(X0[4], oracle.sequential_solve(A, B[4], uplo)) <= TOL
    dX.zero_()
    it, resid = S.solve_batch(dB, dX, mode=1, tol=1e-12, maxit=6)
    assert resid <= 1e-12
    assert max(rel_err(dX.cpu().numpy()[k], Xt[k]) for k in range(9)) <= TOL
    assert S.compact() == 0  # twice is a no-op
    # the paths that read the released pools are refused
    with pytest.raises(SpkError):
        S.set_truncation(-1.0)
    # preprocessing again restores the whole system
    S.preproc(A.a, A.ia, A.ja, A.m, 37, uplo, 1)
    assert S.scalar("lean") == 0 and S.scalar("device_bytes") >= 0.9 * bytes_full
    assert np.array_equal(S.solve(B[0]), x_full)


def test_compact_refused_without_chains():
    L = synth.banded_lower(70000, seed=3)
    S = spk.System().preproc(L.a, L.ia, L.ja, L.m, 16, "L", 1)
    S.set_truncation(-1.0)  # exact mode: the partition solve, no chains
    assert S.scalar("chain") == 0
    with pytest.raises(SpkError):
        S.compact()
