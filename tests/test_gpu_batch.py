"""Batched solves (many right-hand sides per launch) in FP64 and in FP32 with FP64
iterative refinement, against single solves, the sequential FP64 oracle and the
known solutions."""
import numpy as np
import pytest

import oracle
import spike_pstrsv_b200 as spk
from cases import rel_err
from spike_pstrsv_b200 import synth

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda:0")


@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("nrhs", [1, 3, 13, 20, 32, 48, 70])
def test_batch_fp64_matches_single_solves(uplo, nrhs):
    L = synth.banded_lower(60000, seed=11)
    A = L if uplo == "L" else synth.transpose(L)
    Xt, B = synth.make_rhs(A, seed=5, nrhs=nrhs)
    # 512 partitions: groups of 17..32 columns take the right-hand-side-parallel solver
    S = spk.System().preproc(A.a, A.ia, A.ja, A.m, 16 if nrhs <= 16 else 512, uplo, 1)
    dB = _dev(B)
    dX = _dev(np.zeros_like(B))
    it, r = S.solve_batch(dB, dX, mode=0)
    X = dX.cpu().numpy()
    assert r <= 1e-12
    for k in range(nrhs):
        assert rel_err(X[k], S.solve(B[k])) <= 1e-13
        assert rel_err(X[k], oracle.sequential_solve(A, B[k], uplo)) <= 1e-12
        assert rel_err(X[k], Xt[k]) <= 1e-12


@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("nrhs", [1, 5, 16, 27, 32, 40])
def test_batch_fp32_refinement_reaches_fp64_accuracy(uplo, nrhs):
    L = synth.banded_lower(60000, seed=12)
    A = L if uplo == "L" else synth.transpose(L)
    Xt, B = synth.make_rhs(A, seed=6, nrhs=nrhs)
    S = spk.System().preproc(A.a, A.ia, A.ja, A.m, 32 if nrhs <= 16 else 512, uplo, 1)
    dB = _dev(B)
    dX = _dev(np.zeros_like(B))
    it, r = S.solve_batch(dB, dX, mode=1, tol=1e-12, maxit=8)
    X = dX.cpu().numpy()
    assert r <= 1e-12
    assert 1 <= it <= 4
    for k in range(nrhs):
        assert rel_err(X[k], oracle.sequential_solve(A, B[k], uplo)) <= 1e-12
        assert rel_err(X[k], Xt[k]) <= 1e-12


def test_batch_fp32_fixed_iterations_and_poisson():
    L = synth.poisson2d_lower(128)
    Xt, B = synth.make_rhs(L, seed=0, nrhs=4)
    S = spk.System().preproc(L.a, L.ia, L.ja, L.m, 4, "L", 1)
    dB, dX = _dev(B), _dev(np.zeros_like(B))
    it, r = S.solve_batch(dB, dX, mode=1, tol=-1.0, maxit=3)
    assert it == 3 and r <= 1e-12
    assert max(rel_err(dX.cpu().numpy()[k], Xt[k]) for k in range(4)) <= 1e-12


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("nparts", [4, 64, 512])
def test_batch32_wide_couplings_match_single_solves(mode, nparts):
    """Groups of 32 and 25 on the 2-D Poisson factor (couplings 128 rows apart, beyond
    the shared window; truncated spikes at 4 partitions)."""
    L = synth.poisson2d_lower(128)
    Xt, B = synth.make_rhs(L, seed=3, nrhs=57)  # groups of 32 and 25
    S = spk.System().preproc(L.a, L.ia, L.ja, L.m, nparts, "L", 1)
    dB, dX = _dev(B), _dev(np.zeros_like(B))
    it, r = S.solve_batch(dB, dX, mode=mode, tol=1e-12, maxit=8)
    X = dX.cpu().numpy()
    assert r <= 1e-12
    for k in range(57):
        assert rel_err(X[k], S.solve(B[k])) <= (1e-13 if mode == 0 else 1e-11)
        assert rel_err(X[k], Xt[k]) <= 1e-11


def test_batch_rejects_host_arrays_and_bad_leading_dimension():
    L = synth.poisson2d_lower(16)
    S = spk.System().preproc(L.a, L.ia, L.ja, L.m, 2, "L", 1)
    import torch
    B = torch.zeros((2, L.m), dtype=torch.float64)
    with pytest.raises(spk.SpkError):
        S.solve_batch(B, B.clone(), mode=0)
    dB = torch.zeros((2, L.m - 1), dtype=torch.float64, device="cuda:0")
    with pytest.raises(spk.SpkError):
        S.solve_batch(dB, dB.clone(), mode=0)


def test_batch_fp32_after_repreprocessing_the_same_handle():
    """Mixed-precision state (FP32 copies, FP64 diagonal) follows a new matrix
    preprocessed on the same handle."""
    S = spk.System()
    for seed in (31, 32):
        L = synth.banded_lower(40000, seed=seed)
        Xt, B = synth.make_rhs(L, seed=seed, nrhs=32)
        S.preproc(L.a, L.ia, L.ja, L.m, 400, "L", 1)
        dB, dX = _dev(B), _dev(np.zeros_like(B))
        it, r = S.solve_batch(dB, dX, mode=1, tol=1e-12, maxit=8)
        assert r <= 1e-12
        X = dX.cpu().numpy()
        assert max(rel_err(X[k], Xt[k]) for k in range(32)) <= 1e-12


@pytest.mark.parametrize("nparts", [8, 512])
def test_batch_paths_agree(nparts):
    """Few tasks (tile solver groups) and many tasks (right-hand-side-parallel
    groups) give the same FP64 answer."""
    L = synth.banded_lower(50000, seed=41)
    Xt, B = synth.make_rhs(L, seed=41, nrhs=24)
    S = spk.System().preproc(L.a, L.ia, L.ja, L.m, nparts, "L", 1)
    dB, dX = _dev(B), _dev(np.zeros_like(B))
    S.solve_batch(dB, dX, mode=0)
    X = dX.cpu().numpy()
    for k in range(24):
        assert rel_err(X[k], Xt[k]) <= 1e-12
        assert rel_err(X[k], S.solve(B[k])) <= 1e-13


@pytest.mark.parametrize("mode", [0, 1])
def test_batch_with_a_lent_workspace(mode):
    """Work columns carved from caller memory give the same answer as the
    system's own buffers; a workspace below the need is refused."""
    import torch
    L = synth.banded_lower(50000, seed=51)
    Xt, B = synth.make_rhs(L, seed=51, nrhs=24)
    S = spk.System().preproc(L.a, L.ia, L.ja, L.m, 512, "L", 1)
    dB = _dev(B)
    ref = _dev(np.zeros_like(B))
    S.solve_batch(dB, ref, mode=mode, tol=1e-12, maxit=8)
    need = S.workspace_bytes(mode, True)
    ws = torch.empty(need, dtype=torch.uint8, device="cuda:0")
    S.set_workspace(ws)
    dX = _dev(np.zeros_like(B))
    it, r = S.solve_batch(dB, dX, mode=mode, tol=1e-12, maxit=8)
    assert r <= 1e-12
    assert np.array_equal(dX.cpu().numpy(), ref.cpu().numpy())
    S.set_workspace(ws[: need // 2])
    with pytest.raises(spk.SpkError):
        S.solve_batch(dB, dX, mode=mode, tol=1e-12, maxit=8)
    S.set_workspace(None)
    S.solve_batch(dB, dX, mode=mode, tol=1e-12, maxit=8)
    assert rel_err(dX.cpu().numpy()[0], Xt[0]) <= 1e-12
