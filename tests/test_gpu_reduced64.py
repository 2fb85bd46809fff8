"""FP32 + refinement keeps the reduced (boundary) system in FP64: with reduced
rows kept (exact mode, many partitions), the FP32 solve gathers the reduced
unknowns into an FP64 scratch, solves every level there and rounds once.  The
single-system batched solve (tile solver and right-hand-side-parallel solver)
and the many-system group must reach scaled residual 1e-12 and agree with
FP64 to refinement accuracy; the FP32 first pass must already be at FP32
accuracy."""
import numpy as np
import pytest

import spike_pstrsv_b200 as spk
from cases import rel_err
from spike_pstrsv_b200 import group, synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nrhs", [8, 32])
def test_fp32_batch_with_kept_reduced_rows(nrhs):
    import torch

    L = synth.banded_lower(262144, seed=41)
    S = spk.System().preproc(L.a, L.ia, L.ja, L.m, 256, "L", 1)
    S.set_truncation(-1.0)  # exact mode: every reduced row is kept
    assert S.scalar("chain") == 0 and S.scalar("kept_reduced_rows") > 0
    Xt, B = synth.make_rhs(L, seed=41, nrhs=nrhs)
    dB = torch.from_numpy(B).cuda()
    dX = torch.zeros_like(dB)
    S.solve_batch(dB, dX, mode=1, tol=-1.0, maxit=0)  # the FP32 pass alone
    X0 = dX.cpu().numpy()
    assert max(rel_err(X0[k], Xt[k]) for k in range(nrhs)) <= 1e-5
    dX.zero_()
    it, resid = S.solve_batch(dB, dX, mode=1, tol=1e-12, maxit=6)
    assert resid <= 1e-12
    X = dX.cpu().numpy()
    assert max(rel_err(X[k], Xt[k]) for k in range(nrhs)) <= 1e-12
    dX.zero_()
    S.solve_batch(dB, dX, mode=0)
    assert max(rel_err(X[k], dX.cpu().numpy()[k]) for k in range(nrhs)) <= 1e-12


def test_group_fp32_with_kept_reduced_rows():
    import torch

    mats, nrhs, rhs = group.build(6, seed=7, m_lo=20000, m_hi=60000)
    systems = []
    for L in mats:
        S = spk.System().preproc(L.a, L.ia, L.ja, L.m, max(16, L.m // 1024), "L", 1)
        S.set_truncation(-1.0)
        systems.append(S)
    assert any(S.scalar("kept_reduced_rows") > 0 for S in systems)
    B = [torch.from_numpy(b).cuda() for _, b in rhs]
    X = [torch.zeros_like(b) for b in B]
    st = torch.cuda.Stream()
    g = group.Group(systems, B, X, mode=group.MODE_FP32_IR, iters=2, stream=st.cuda_stream)
    g.solve()
    st.synchronize()
    assert g.residual() <= 1e-12
    for (xt, _), x in zip(rhs, X):
        assert rel_err(x.cpu().numpy(), xt) <= 1e-11
