"""The error path of the bounded device waits, driven by a test hook instead of a
real hang: with spk_debug_set(s, "fail_waits", 1) every solve kernel reports a
failed wait at entry, before it issues any copy, and returns.  The synchronous
solve must surface SPK_ERR_TIMEOUT, and the next solve must run normally on the
same system (the context stays usable, the error word is cleared)."""
import numpy as np
import pytest

import spike_pstrsv_b200 as spk
from cases import rel_err
from spike_pstrsv_b200 import synth

pytestmark = pytest.mark.gpu
TIMEOUT = -7


def _system(monkeypatch, chain):
    monkeypatch.setenv("SPK_DISABLE_CHAIN", "0" if chain else "1")
    L = synth.banded_lower(65536, seed=4)
    x_true, b = synth.make_rhs(L, seed=4)
    S = spk.System().preproc(L.a, L.ia, L.ja, L.m, 16, "L", 1)
    assert S.scalar("chain") == int(chain)
    return L, S, x_true, b


@pytest.mark.parametrize("chain", [True, False], ids=["chain", "partitions"])
def test_plain_solve_reports_failed_wait_then_recovers(monkeypatch, chain):
    L, S, x_true, b = _system(monkeypatch, chain)
    S.debug_set("fail_waits", 1)
    with pytest.raises(spk.SpkError) as e:
        S.solve(b)
    assert e.value.code == TIMEOUT
    x = S.solve(b)  # the hook ended with the reported failure
    assert rel_err(x, x_true) <= 1e-12


def test_batched_solve_reports_failed_wait_then_recovers(monkeypatch):
    import torch

    L, S, _, _ = _system(monkeypatch, False)
    Xt, B = synth.make_rhs(L, seed=6, nrhs=4)
    dB = torch.from_numpy(B).cuda()
    dX = torch.zeros_like(dB)
    S.debug_set("fail_waits", 1)
    with pytest.raises(spk.SpkError) as e:
        S.solve_batch(dB, dX, mode=0)
    assert e.value.code == TIMEOUT
    S.solve_batch(dB, dX, mode=0)
    X = dX.cpu().numpy()
    assert max(rel_err(X[k], Xt[k]) for k in range(4)) <= 1e-12


def test_async_solve_failure_is_reported_by_check(monkeypatch):
    import torch

    L, S, x_true, b = _system(monkeypatch, True)
    db = torch.from_numpy(b).cuda()
    dx = torch.zeros_like(db)
    sp = torch.cuda.current_stream().cuda_stream
    S.debug_set("fail_waits", 1)
    S.solve_device(db.data_ptr(), dx.data_ptr(), sp)
    with pytest.raises(spk.SpkError) as e:
        S.check()
    assert e.value.code == TIMEOUT
    S.check()  # reported once; nothing pending
    S.solve_device(db.data_ptr(), dx.data_ptr(), sp)
    S.check()
    assert rel_err(dx.cpu().numpy(), x_true) <= 1e-12


def test_unknown_debug_setting_is_refused():
    L = synth.banded_lower(4096, seed=1)
    S = spk.System().preproc(L.a, L.ia, L.ja, L.m, 4, "L", 1)
    with pytest.raises(spk.SpkError) as e:
        S.debug_set("no_such_setting", 1)
    assert e.value.code == -1
    assert np.isfinite(S.solve(synth.make_rhs(L, seed=1)[1])).all()
