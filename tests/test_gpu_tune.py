"""Chain-solver knobs (spk_tune) and the per-system autotuner: every setting
still solves to the sequential FP64 oracle within 1e-12, the tuner keeps its
fastest candidate, invalid settings are rejected."""
import numpy as np
import pytest

import oracle
import spike_pstrsv_b200 as spk
from cases import rel_err
from spike_pstrsv_b200 import synth, tune
from spike_pstrsv_b200.capi import SpkError

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _system(m=200000, uplo="L"):
    L = synth.banded_lower(m, seed=21)
    A = L if uplo == "L" else synth.transpose(L)
    S = spk.System().preproc(A.a, A.ia, A.ja, A.m, 64, uplo, 1)
    assert S.scalar("chain") == 1
    return A, S


@pytest.mark.parametrize("uplo", ["L", "U"])
def test_knobs_keep_results(uplo):
    import torch

    A, S = _system(uplo=uplo)
    _, b = synth.make_rhs(A, seed=3)
    xo = oracle.sequential_solve(A, b, uplo)
    rows0 = S.scalar("rows")
    for rows in (rows0 // 2, rows0 * 2):
        S.tune("rows", rows)
        assert S.scalar("rows") >= 32 * ((rows + 31) // 32)
        for stages in (2, 3):
            S.tune("stages", stages)
            assert S.scalar("stages") == stages
            assert rel_err(S.solve(b), xo) <= TOL
    Xt, B = synth.make_rhs(A, seed=4, nrhs=20)
    dB = torch.from_numpy(B).cuda()
    for path, rows in ((1, S.scalar("batch_rows") // 2), (1, S.scalar("batch_rows") * 2), (0, None)):
        if rows:
            S.tune("batch_rows", rows)
        S.tune("batch_path", path)
        assert S.scalar("batch_path") == path
        for mode in (0, 1):
            dX = torch.zeros_like(dB)
            _, r = S.solve_batch(dB, dX, mode=mode, tol=1e-12, maxit=8)
            X = dX.cpu().numpy()
            assert r <= TOL
            for k in (0, 7, 19):
                assert rel_err(X[k], oracle.sequential_solve(A, B[k], uplo)) <= TOL, (path, rows, mode, k)


def test_knobs_reject_bad_values_and_reset_on_preprocessing():
    A, S = _system(m=50000)
    for name, v in (("stages", 4), ("rows", 8), ("batch_path", 2), ("nonsense", 1)):
        with pytest.raises(SpkError):
            S.tune(name, v)
    S.tune("batch_path", 0).tune("stages", 3)
    S.preproc(A.a, A.ia, A.ja, A.m, 64, "L", 1)
    assert S.scalar("batch_path") == -1 and S.scalar("stages") == 2
    S.compact()
    with pytest.raises(SpkError):
        S.tune("batch_path", 0)  # the partition pools were released
    S.tune("batch_path", 1)


def test_autotuner_keeps_the_fastest_setting():
    import torch

    A, S = _system()
    Xt, b = synth.make_rhs(A, seed=5)
    db = torch.from_numpy(b).cuda()
    dx = torch.zeros_like(db)
    res = tune.tune_solve(S, db, dx, reps=5)
    best = min(res["ms"], key=res["ms"].get)
    assert (res["choice"]["rows"], res["choice"]["stages"]) == best
    assert (S.scalar("rows"), S.scalar("stages")) == best
    assert rel_err(S.solve(b), oracle.sequential_solve(A, b, "L")) <= TOL
    _, B = synth.make_rhs(A, seed=6, nrhs=16)
    dB = torch.from_numpy(B).cuda()
    dX = torch.zeros_like(dB)
    rb = tune.tune_batch(S, dB, dX, mode=0, reps=2)
    path, rows = min(rb["ms"], key=rb["ms"].get)
    assert rb["choice"]["path"] == path
    assert S.scalar("batch_path") == (1 if path == "chain" else 0)
    dX.zero_()
    _, r = S.solve_batch(dB, dX, mode=0, tol=1e-12, maxit=4)
    assert r <= TOL
    assert rel_err(dX.cpu().numpy()[3], oracle.sequential_solve(A, B[3], "L")) <= TOL
