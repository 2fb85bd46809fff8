"""Many systems in one captured launch sequence: every system's columns against
x_true, the sequential FP64 oracle and its own batched solve, FP64 and FP32 +
refinement, graph replays, the autotuner, error paths."""
import numpy as np
import pytest

import oracle
import spike_pstrsv_b200 as spk
from spike_pstrsv_b200 import group, synth
from spike_pstrsv_b200.capi import SpkError

pytestmark = pytest.mark.gpu


def _pool(count, seed):
    mats, nrhs, rhs = group.build(count, seed=seed, m_lo=1024, m_hi=30000)
    return mats, nrhs, rhs


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("mode,iters", [(group.MODE_FP64, 0), (group.MODE_FP32_IR, 2)])
def test_group_matches_each_system(mode, iters):
    import torch
    mats, nrhs, rhs = _pool(20, seed=3)
    systems = [spk.System().preproc(L.a, L.ia, L.ja, L.m, max(2, L.m // 2048), "L", 1) for L in mats]
    B = [torch.from_numpy(b).cuda() for _, b in rhs]
    X = [torch.zeros_like(b) for b in B]
    st = torch.cuda.Stream()
    g = group.Group(systems, B, X, mode=mode, iters=iters, stream=st.cuda_stream)
    assert g.info("columns") == sum(nrhs)
    assert g.info("kernels") >= 2
    for rep in range(2):  # two replays of the captured graph
        for x in X:
            x.zero_()
        torch.cuda.synchronize()
        g.solve()
        st.synchronize()
        assert g.residual() <= 1e-12
        for i, ((Xt, Bh), x) in enumerate(zip(rhs, X)):
            xx = x.cpu().numpy()
            assert _rel(xx, Xt) <= 1e-11
            ref = torch.zeros_like(B[i])
            systems[i].solve_batch(B[i], ref, mode=0, want_resid=False)
            assert _rel(xx, ref.cpu().numpy()) <= 1e-12
            if rep == 0:
                xo = np.stack([oracle.sequential_solve(mats[i], Bh[k], "L") for k in range(Bh.shape[0])])
                assert _rel(xx, xo) <= 1e-12
    g.close()


def test_group_rejects_default_stream_and_bad_members():
    import torch
    L = synth.poisson_banded_lower(5000, 8.0, 64, seed=1)
    S = spk.System().preproc(L.a, L.ia, L.ja, L.m, 4, "L", 1)
    B = [torch.zeros((2, L.m), dtype=torch.float64, device="cuda")]
    X = [torch.zeros_like(B[0])]
    with pytest.raises(SpkError):
        group.Group([S], B, X, stream=0)  # the legacy default stream cannot be captured
    Bs = [torch.zeros((2, L.m - 1), dtype=torch.float64, device="cuda")]
    with pytest.raises(SpkError):
        group.Group([S], Bs, X, stream=torch.cuda.Stream().cuda_stream)


def test_autotune_picks_a_partition_size_per_class():
    mats, nrhs, _ = _pool(6, seed=5)
    choice, table = group.autotune(mats, nrhs, candidates=(512, 2048, 8192), reps=2)
    assert set(choice) == {group.size_class(L.m) for L in mats}
    for c, rows in choice.items():
        assert rows in (512, 2048, 8192)
        assert min(table[c]["seconds"].values()) == table[c]["seconds"][rows]
