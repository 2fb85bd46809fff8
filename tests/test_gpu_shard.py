"""The phases of the sharded chain solve on one GPU: every rank of an emulated
world of 2 and 3 ranks has its own x buffer; ranks run phase 1 (spk_chain_phase)
one after another, the halo rows are copied from the next rank's buffer as the
point-to-point exchange would deliver them, and each rank runs phase 4.  The
rows each rank owns, assembled, must equal the single-GPU solve (no kernel
waits for another: the emulation runs the ranks' launches in sequence)."""
import numpy as np
import pytest

import spike_pstrsv_b200 as spk
from cases import rel_err
from spike_pstrsv_b200 import shard, synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("uplo", ["L", "U"])
def test_emulated_ranks_match_single_gpu(world, uplo):
    import torch

    L = synth.banded_lower(300000, seed=31)
    A = L if uplo == "L" else synth.transpose(L)
    x_true, b = synth.make_rhs(A, seed=31)
    S = spk.System().preproc(A.a, A.ia, A.ja, A.m, 64, uplo, 1)
    assert S.scalar("chain") == 1
    db = torch.from_numpy(b).cuda()
    ref = torch.zeros_like(db)
    S.solve(db, ref)
    n, reach, rev = A.m, S.scalar("chain_reach"), uplo == "L"
    tasks = S.array("chain_tasks1")
    ranges = shard.plan(tasks, world)
    xs = [torch.full_like(db, float("nan")) for _ in range(world)]
    sp = torch.cuda.current_stream().cuda_stream
    for r, (lo, hi) in enumerate(ranges):
        S.chain_phase(1, lo, hi, db.data_ptr(), xs[r].data_ptr(), sp)
    for r, (lo, hi) in enumerate(ranges):
        if r + 1 < world:
            sl = shard.caller_slice(n, rev, hi, hi + reach)
            xs[r][sl] = xs[r + 1][sl]
    for r, (lo, hi) in enumerate(ranges):
        S.chain_phase(4, lo, hi, db.data_ptr(), xs[r].data_ptr(), sp)
    S.check()
    x = torch.full_like(db, float("nan"))
    for r, (lo, hi) in enumerate(ranges):
        sl = shard.caller_slice(n, rev, lo, hi)
        x[sl] = xs[r][sl]
    xh = x.cpu().numpy()
    assert np.isfinite(xh).all()
    assert rel_err(xh, ref.cpu().numpy()) <= 1e-15
    assert rel_err(xh, x_true) <= 1e-12


def test_chain_phase_is_refused_without_chains():
    L = synth.banded_lower(20000, seed=2)
    S = spk.System().preproc(L.a, L.ia, L.ja, L.m, 8, "L", 1).set_truncation(-1.0)
    import torch

    db = torch.zeros(L.m, dtype=torch.float64, device="cuda")
    with pytest.raises(spk.SpkError) as e:
        S.chain_phase(1, 0, L.m, db.data_ptr(), db.data_ptr())
    assert e.value.code == -5
