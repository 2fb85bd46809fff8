"""Serving loop: every result is the same alone and in a concurrent mix (scaled
residual <= 1e-12, alone vs mix and against the sequential FP64 oracle within
1e-12 relative), LRU eviction under a
small HBM budget, continuous batching of queued requests, error paths."""
import threading

import numpy as np
import pytest

import oracle
from spike_pstrsv_b200 import serve, synth
from spike_pstrsv_b200.capi import SpkError

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _pool(count=4, seed=0):
    rng = np.random.default_rng(seed)
    mats = []
    for i in range(count):
        m = int(rng.integers(20000, 90000))
        band = int(rng.integers(32, 129))
        L = synth.poisson_banded_lower(m, 8.0, band, seed=100 + i)
        mats.append(L)
    return mats


def _requests(mats, count, seed):
    rng = np.random.default_rng(seed)
    reqs = []
    for j in range(count):
        mid = int(rng.integers(len(mats)))
        k = int(rng.choice([1, 2, 4, 8, 16]))
        Xt, B = synth.make_rhs(mats[mid], seed=1000 + j, nrhs=k)
        reqs.append((mid, B, Xt))
    return reqs


@pytest.mark.parametrize("mode", [serve.MODE_FP32_IR, serve.MODE_FP64])
def test_results_are_the_same_alone_and_in_the_mix(mode):
    mats = _pool()
    reqs = _requests(mats, 24, seed=mode)
    with serve.Server(hbm_budget_bytes=8 << 30, slots=3) as S:
        for i, L in enumerate(mats):
            S.put_matrix(i, L.a, L.ia, L.ja, L.m, 8, "L")
        alone = []
        for mid, B, Xt in reqs:
            r = S.submit(mid, B, mode).wait()
            assert r.batch_rhs == B.shape[0]
            alone.append(r.x.copy())
        # the mix: four client threads submit interleaved, then wait
        tickets = [None] * len(reqs)

        def client(c):
            for j in range(c, len(reqs), 4):
                tickets[j] = S.submit(reqs[j][0], reqs[j][1], mode)

        th = [threading.Thread(target=client, args=(c,)) for c in range(4)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        mixed = [t.wait() for t in tickets]
        st = S.stats()
    assert max(r.batch_rhs for r in mixed) > min(B.shape[0] for _, B, _ in reqs)  # requests were batched
    for (mid, B, Xt), a, r in zip(reqs, alone, mixed):
        if mode == serve.MODE_FP32_IR:
            assert 0 <= r.scaled_residual <= TOL
        assert _rel(r.x, a) <= TOL
        assert _rel(r.x, Xt) <= 1e-11
        xo = np.stack([oracle.sequential_solve(mats[mid], B[k], "L") for k in range(B.shape[0])])
        assert _rel(r.x.reshape(xo.shape), xo) <= TOL
        assert r.latency_s > 0
    assert st["completed"] == 2 * len(reqs)
    assert st["preprocessings"] == len(mats)


def _footprints(mats, P=8):
    """Device bytes of each matrix's system, whole and compacted (spk_compact)."""
    from spike_pstrsv_b200.capi import System

    full, lean = [], []
    for L in mats:
        S = System().preproc(L.a, L.ia, L.ja, L.m, P, "L", 1)
        full.append(S.scalar("device_bytes"))
        S.compact()
        lean.append(S.scalar("device_bytes"))
        S.close()
    return full, lean


def test_idle_systems_are_compacted_before_any_eviction():
    mats = _pool(count=4, seed=5)
    full, lean = _footprints(mats)
    # every system fits once compacted, not all of them whole
    budget = sum(lean) + (sum(full) - sum(lean)) // 2 + (48 << 20)
    with serve.Server(hbm_budget_bytes=budget, slots=1) as S:
        for i, L in enumerate(mats):
            S.put_matrix(i, L.a, L.ia, L.ja, L.m, 8, "L")
        for rnd in range(2):
            for i, L in enumerate(mats):
                Xt, B = synth.make_rhs(L, seed=11 * i + rnd, nrhs=4)
                for mode in (serve.MODE_FP32_IR, serve.MODE_FP64):
                    r = S.submit(i, B, mode).wait()
                    assert r.scaled_residual <= TOL
                    assert _rel(r.x, Xt) <= 1e-11
        st = S.stats()
    assert st["compactions"] > 0
    assert st["resident_bytes"] <= budget


def test_lru_eviction_under_a_small_budget():
    mats = _pool(count=4, seed=3)
    full, lean = _footprints(mats)
    # room for about two resident systems, even compacted, with their batch buffers
    with serve.Server(hbm_budget_bytes=sum(lean) // 2 + (24 << 20), slots=2) as S:
        for i, L in enumerate(mats):
            S.put_matrix(i, L.a, L.ia, L.ja, L.m, 8, "L")
        for rnd in range(2):
            for i, L in enumerate(mats):
                Xt, B = synth.make_rhs(L, seed=7 * i + rnd, nrhs=4)
                r = S.submit(i, B, serve.MODE_FP32_IR).wait()
                assert r.scaled_residual <= TOL
                assert _rel(r.x, Xt) <= 1e-11
        st = S.stats()
    assert st["evictions"] > 0
    assert st["preprocessings"] > len(mats)
    assert st["resident_systems"] < len(mats)


def test_queued_requests_of_one_matrix_share_a_batch():
    L = synth.poisson_banded_lower(200000, 8.0, 64, seed=5)
    with serve.Server(hbm_budget_bytes=8 << 30, slots=1) as S:
        S.put_matrix(0, L.a, L.ia, L.ja, L.m, 64, "L")
        S.submit(0, synth.make_rhs(L, seed=0)[1], serve.MODE_FP64).wait()  # preprocessed
        sols = [synth.make_rhs(L, seed=s) for s in range(1, 41)]
        tickets = [S.submit(0, B, serve.MODE_FP64) for _, B in sols]
        res = [t.wait() for t in tickets]
        st = S.stats()
    assert max(r.batch_rhs for r in res) >= 8
    assert st["batches"] < 41
    for (Xt, _), r in zip(sols, res):
        assert _rel(r.x[0], Xt) <= 1e-11


def test_server_errors():
    L = synth.poisson2d_lower(32)
    with serve.Server(hbm_budget_bytes=1 << 30, slots=1) as S:
        S.put_matrix(0, L.a, L.ia, L.ja, L.m, 2, "L")
        with pytest.raises(ValueError):
            S.submit(0, np.zeros(L.m + 1))
        with pytest.raises(SpkError):
            serve._bind()
            S.n[5] = L.m
            S.submit(5, np.zeros(L.m))
        with pytest.raises(SpkError):
            S.put_matrix(1, L.a, L.ia, L.ja, L.m, L.m + 1, "L")
        _, B = synth.make_rhs(L, seed=0)
        r = S.submit(0, B).wait()
        assert r.scaled_residual <= TOL


def test_batches_above_the_tolerance_are_solved_again_in_fp64():
    """Values beyond the FP32 range (|a| ~ 1e39): the FP32 solve overflows, its
    residual is NaN (not 'converged'), and the server re-solves the batch in FP64,
    which meets the tolerance."""
    n = 64
    ia = np.zeros(n + 1, dtype=np.int32)
    ja, a = [], []
    for i in range(n):
        if i:
            ja.append(i - 1)
            a.append(-1e38)
        ja.append(i)
        a.append(1e39)
        ia[i + 1] = len(ja)
    L = synth.CSR(n, ia, np.asarray(ja, np.int32), np.asarray(a))
    Xt, B = synth.make_rhs(L, seed=0, nrhs=2)
    with serve.Server(hbm_budget_bytes=1 << 30, slots=1) as S:
        S.put_matrix(0, L.a, L.ia, L.ja, n, 2, "L")
        r = S.submit(0, B, serve.MODE_FP32_IR).wait()
        st = S.stats()
    assert st["rechecks"] >= 1
    assert 0 <= r.scaled_residual <= TOL
    assert _rel(r.x, Xt) <= 1e-12


def test_fp32_batch_reports_a_nan_residual_when_the_values_overflow():
    import torch
    import spike_pstrsv_b200 as spk
    n = 64
    ia = np.concatenate([[0], np.cumsum([1] + [2] * (n - 1))]).astype(np.int32)
    ja = np.concatenate([[0]] + [[i - 1, i] for i in range(1, n)]).astype(np.int32)
    a = np.concatenate([[1e39]] + [[-1e38, 1e39] for _ in range(1, n)])
    L = synth.CSR(n, ia, ja, a)
    _, B = synth.make_rhs(L, seed=1, nrhs=3)
    S = spk.System().preproc(L.a, L.ia, L.ja, n, 2, "L", 1)
    dB = torch.from_numpy(B).cuda()
    dX = torch.zeros_like(dB)
    it, r = S.solve_batch(dB, dX, mode=1, tol=1e-12, maxit=3)
    assert not (r <= 1e-12)  # NaN or large: never reported as converged
    it, r = S.solve_batch(dB, dX, mode=0)
    assert r <= 1e-12
