"""The chain solver (the default one-right-hand-side solve when spike truncation
is on) against the sequential FP64 substitution, x_true and the partition-based
solve it replaces.

Rows are cut into chains independent of the partition count; every chain's
spike is computed at preprocessing and decides which rows phase 4 re-solves
(chain.cu).  The reference state (partitions, pools, spikes, reduced system) is
untouched, so the structure tests in test_gpu_parity.py hold as before."""
import numpy as np
import pytest

import oracle
import spike_pstrsv_b200 as spk
from cases import random_cases, rel_err
from spike_pstrsv_b200 import synth

pytestmark = pytest.mark.gpu
TOL = 1e-12


def gpu_system(A, P, uplo, flb=1):
    return spk.System().preproc(A.a, A.ia, A.ja, A.m, P, uplo, flb)


@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("P", [1, 4, 64, 300])
def test_chain_engages_and_matches_substitution(uplo, P):
    L = synth.banded_lower(262144, seed=5)
    A = L if uplo == "L" else synth.transpose(L)
    x_true, b = synth.make_rhs(A, seed=5)
    S = gpu_system(A, P, uplo)
    assert S.scalar("chain") == 1
    assert S.scalar("chains") >= 64                     # parallelism no longer set by P
    assert S.scalar("chain_rows_phase4") < A.m // 2     # only the coupled rows are re-solved
    x = S.solve(b)
    xs = oracle.sequential_solve(A, b, uplo)
    assert rel_err(x, xs) <= TOL
    assert rel_err(x, x_true) <= TOL


def test_chain_agrees_with_partition_solve(monkeypatch):
    L = synth.banded_lower(200000, seed=7)
    x_true, b = synth.make_rhs(L, seed=7)
    S = gpu_system(L, 64, "L")
    assert S.scalar("chain") == 1
    monkeypatch.setenv("SPK_DISABLE_CHAIN", "1")
    Q = gpu_system(L, 64, "L")
    assert Q.scalar("chain") == 0
    x, xq = S.solve(b), Q.solve(b)
    assert rel_err(x, xq) <= 1e-15
    E = gpu_system(L, 64, "L").set_truncation(-1.0)      # exact mode: reference phases, no chains
    assert E.scalar("chain") == 0
    assert rel_err(x, E.solve(b)) <= 1e-15


@pytest.mark.parametrize("m", [100003, 4097, 1000])
def test_chain_ragged_sizes(m):
    """Row counts that are not multiples of the 32-row tile, and small systems
    (which may keep the partition-based solve)."""
    L = synth.banded_lower(m, seed=m)
    x_true, b = synth.make_rhs(L, seed=1)
    for uplo, A in (("L", L), ("U", synth.transpose(L))):
        bb = b if uplo == "L" else synth.spmv(A, x_true)
        S = gpu_system(A, 8, uplo)
        x = S.solve(bb)
        assert rel_err(x, oracle.sequential_solve(A, bb, uplo)) <= TOL, (uplo, S.scalar("chain"))


@pytest.mark.parametrize("rows", [1024, 2048, 8192])
def test_chain_lengths(monkeypatch, rows):
    """Chains of several lengths (the length is doubled at preprocessing until
    every chain keeps its first rows final)."""
    monkeypatch.setenv("SPK_CHAIN_ROWS", str(rows))
    L = synth.banded_lower(150000, seed=11)
    x_true, b = synth.make_rhs(L, seed=11)
    S = gpu_system(L, 16, "L")
    assert S.scalar("chain") == 1 and S.scalar("chain_rows") >= rows
    assert rel_err(S.solve(b), oracle.sequential_solve(L, b, "L")) <= TOL


def test_chain_poisson_and_random():
    """Inputs whose spikes decay slowly or not at all, and irregular random
    matrices: whichever path preprocessing picks, x matches the substitution."""
    L = synth.poisson2d_lower(128)
    x_true, b = synth.make_rhs(L, seed=0)
    for P in (1, 4, 16):
        S = gpu_system(L, P, "L")
        assert rel_err(S.solve(b), oracle.sequential_solve(L, b, "L")) <= TOL
    for name, A, P in random_cases(12, base_seed=77):
        S = gpu_system(A, P, "U")
        _, bb = synth.make_rhs(A, seed=3)
        assert rel_err(S.solve(bb), oracle.sequential_solve(A, bb, "U")) <= TOL, name


def test_chain_repeat_and_legacy_api():
    """Repeated solves are identical (no state kept between calls) and the
    reference-facing entry point (host arrays: copies overlapped with the chain
    kernels) gives the same x."""
    L = synth.banded_lower(131072, seed=2)
    x_true, b = synth.make_rhs(L, seed=2)
    S = gpu_system(L, 32, "L")
    x1 = S.solve(b)
    x2 = S.solve(b)
    assert np.array_equal(x1, x2)
    spk.spike_pstrsv_preproc(L.a, L.ia, L.ja, L.m, 32, "L")
    for _ in range(2):
        x = np.zeros(L.m)
        spk.spike_pstrsv_solve("L", L.m, b.copy(), x, 32)
        assert rel_err(x, x1) <= 1e-15


@pytest.mark.parametrize("chunks", ["1", "3", "64"])
def test_pipelined_host_solve(monkeypatch, chunks):
    """The host-array solve in 1, 3 and 64 copy chunks (page-locked and pageable
    buffers) against the device-resident solve, 'L' and 'U'."""
    import torch

    monkeypatch.setenv("SPK_PIPELINE_CHUNKS", chunks)
    L = synth.banded_lower(300000, seed=8)
    for uplo, A in (("L", L), ("U", synth.transpose(L))):
        x_true, b = synth.make_rhs(A, seed=8)
        S = gpu_system(A, 16, uplo)
        assert S.scalar("chain") == 1
        db = torch.from_numpy(b).cuda()
        dx = torch.zeros_like(db)
        S.solve(db, dx)
        xd = dx.cpu().numpy()
        bh = torch.from_numpy(b).pin_memory()
        xh = torch.zeros(A.m, dtype=torch.float64).pin_memory()
        S.solve(bh.numpy(), xh.numpy())
        assert np.array_equal(xh.numpy(), xd)
        assert np.array_equal(S.solve(b), xd)
        assert rel_err(xd, x_true) <= TOL


@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("nrhs", [1, 5, 32, 40])
def test_chain_batched_matches_substitution(monkeypatch, uplo, nrhs):
    """Batched solves through the right-hand-side-parallel chain kernel (lane =
    right-hand side): FP64 against the sequential substitution of every column,
    FP32 + FP64 refinement to scaled residual 1e-12."""
    import torch

    monkeypatch.setenv("SPK_CHAIN_BATCH", "1")  # the chain kernels whatever the partition count
    L = synth.banded_lower(120000, seed=12)
    A = L if uplo == "L" else synth.transpose(L)
    Xt, B = synth.make_rhs(A, seed=12, nrhs=nrhs)
    S = gpu_system(A, 8, uplo)
    assert S.scalar("chain") == 1
    dB = torch.from_numpy(B).cuda()
    dX = torch.zeros_like(dB)
    S.solve_batch(dB, dX, mode=0)
    X = dX.cpu().numpy()
    for k in range(nrhs):
        assert rel_err(X[k], oracle.sequential_solve(A, B[k], uplo)) <= TOL, k
    dX.zero_()
    it, resid = S.solve_batch(dB, dX, mode=1, tol=1e-12, maxit=6)
    assert resid <= 1e-12 and it >= 1
    X = dX.cpu().numpy()
    assert max(rel_err(X[k], Xt[k]) for k in range(nrhs)) <= TOL


@pytest.mark.parametrize("per_row,band,m", [(1, 8, 70001), (3, 16, 65539), (7, 128, 90013),
                                            (24, 100, 100003), (33, 64, 200003)])
def test_chain_batched_widths(monkeypatch, per_row, band, m):
    """The batched chain kernel at every slot width (4 to 64 slots per tile),
    reach up to 128 and row counts that are not a multiple of the 32-row tile
    (so a task's first tile starts part-way), FP64 against the substitution."""
    import torch

    monkeypatch.setenv("SPK_CHAIN_BATCH", "1")
    L = synth.banded_lower(m, per_row=per_row, band=band, seed=per_row)
    for uplo in ("L", "U"):
        A = L if uplo == "L" else synth.transpose(L)
        Xt, B = synth.make_rhs(A, seed=3, nrhs=7)
        S = gpu_system(A, 16, uplo)
        assert S.scalar("chain") == 1
        dB = torch.from_numpy(B).cuda()
        dX = torch.zeros_like(dB)
        S.solve_batch(dB, dX, mode=0)
        X = dX.cpu().numpy()
        for k in (0, 3, 6):
            assert rel_err(X[k], oracle.sequential_solve(A, B[k], uplo)) <= TOL, (uplo, k)
        assert max(rel_err(X[k], Xt[k]) for k in range(7)) <= TOL
        # the single solve (lane = row kernel) agrees to rounding
        assert rel_err(S.solve(B[2]), X[2]) <= 1e-14


@pytest.mark.parametrize("chunks", ["4", "16"])
def test_pipelined_host_solve_replays_its_graph(monkeypatch, chunks):
    """Repeated host-array solves on the same page-locked b and x replay the
    pipeline captured on the second call: every result equals the device
    solve's, new contents of the same buffers are read at each replay, other
    buffers and a re-preprocessed system give a fresh pipeline."""
    import torch

    monkeypatch.setenv("SPK_PIPELINE_CHUNKS", chunks)
    L = synth.banded_lower(300007, seed=31)
    S = gpu_system(L, 64, "L")
    hb = torch.empty(L.m, dtype=torch.float64).pin_memory()
    hx = torch.empty(L.m, dtype=torch.float64).pin_memory()
    for rep in range(5):
        xt, b = synth.make_rhs(L, seed=100 + rep)
        hb.numpy()[:] = b
        hx.zero_()
        S.solve(hb.numpy(), hx.numpy())
        xd = torch.empty(L.m, dtype=torch.float64, device="cuda")
        S.solve_device(torch.from_numpy(b).cuda().data_ptr(), xd.data_ptr())
        assert np.array_equal(hx.numpy(), xd.cpu().numpy()), rep
        assert rel_err(hx.numpy(), xt) <= TOL
    hb2 = torch.from_numpy(b.copy()).pin_memory()
    hx2 = torch.zeros(L.m, dtype=torch.float64).pin_memory()
    S.solve(hb2.numpy(), hx2.numpy())
    assert np.array_equal(hx2.numpy(), hx.numpy())
    # another matrix under the same buffers
    L2 = synth.banded_lower(300007, per_row=8, band=40, seed=32)
    S.preproc(L2.a, L2.ia, L2.ja, L2.m, 64, "L", 1)
    for rep in range(3):
        xt2, b2 = synth.make_rhs(L2, seed=200 + rep)
        hb.numpy()[:] = b2
        S.solve(hb.numpy(), hx.numpy())
        assert rel_err(hx.numpy(), oracle.sequential_solve(L2, b2, "L")) <= TOL
