"""CUDA path against the oracle and the reference's golden fixtures.

Structure (partitions, flags, intervals, every CSR pool, mapR, the dense spikes
S and the reduced system T) must be bit-identical; x must agree to relative
error <= 1e-12 (the reference's own solve is only tolerance-deterministic,
src/spike_pstrsv.c:213-229)."""
import glob
import hashlib
import json
import os

import numpy as np
import pytest

import oracle
import spike_pstrsv_b200 as spk
from cases import random_cases, rel_err, struct_diff
from spike_pstrsv_b200 import synth
from test_oracle_pins import DIGEST, GOLDEN, load_small, make_case, sha, trim_S

pytestmark = pytest.mark.gpu
TOL = 1e-12


def gpu_system(A, P, uplo, flb):
    return spk.System().preproc(A.a, A.ia, A.ja, A.m, P, uplo, flb)


SMALL = sorted(glob.glob(os.path.join(GOLDEN, "small_*.npz")))


@pytest.mark.parametrize("path", SMALL, ids=[os.path.basename(p)[6:-4] for p in SMALL])
def test_gpu_matches_golden_small(path):
    A, P, flb, uplo, b, x_ref, want = load_small(path)
    S = gpu_system(A, P, uplo, flb)
    got = trim_S(S.structure(), len(want["S"]))
    assert struct_diff(got, want) == []
    assert rel_err(S.solve(b), x_ref) <= TOL


@pytest.mark.parametrize("name", sorted(k for k, v in DIGEST.items() if v["m"] <= 65536))
def test_gpu_matches_golden_digest(name):
    rec = DIGEST[name]
    A = make_case(rec)
    S = gpu_system(A, rec["P"], rec["uplo"], rec["flb"])
    got = trim_S(S.structure(), rec["sizes"]["S"])
    bad = [k for k, h in rec["arrays"].items() if sha(got[k]) != h]
    bad += [k for k, v in rec["scalars"].items() if int(got[k]) != v]
    assert bad == []
    x_true, b = synth.make_rhs(A, seed=0)
    x = S.solve(b)
    xs = oracle.sequential_solve(A, b, rec["uplo"])
    assert rel_err(x, xs) <= TOL
    assert rel_err(x, x_true) <= TOL


@pytest.mark.parametrize("flb", [0, 1])
def test_gpu_matches_oracle_random(flb):
    failures = []
    for name, A, P in random_cases(40):
        O = oracle.Oracle()
        assert O.preproc(A, P, uplo="U", flb=flb) == 0
        want = O.structure()
        S = gpu_system(A, P, "U", flb)
        bad = struct_diff(S.structure(), want)
        _, b = synth.make_rhs(A, seed=1)
        err = rel_err(S.solve(b), O.solve(b))
        if bad or err > TOL:
            failures.append((name, bad, err))
    assert failures == []


@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("P", [1, 2, 4, 16])
def test_legacy_api_host_pointers(uplo, P):
    L = synth.poisson2d_lower(128)
    A = L if uplo == "L" else synth.transpose(L)
    x_true, b = synth.make_rhs(A, seed=0)
    b0 = b.copy()
    x = np.zeros(A.m)
    spk.spike_pstrsv_preproc(A.a, A.ia, A.ja, A.m, P, uplo)
    spk.spike_pstrsv_solve(uplo, A.m, b, x, P)
    assert np.array_equal(b, b0)  # b is left unchanged unless SPK_CLOBBER_B is set
    O = oracle.Oracle()
    O.preproc(A, P, uplo=uplo, flb=1)
    assert struct_diff(spk.legacy_structure(), O.structure()) == []
    assert spk.get_global("numRowsReducedSystem") == O.scalar("numRowsReducedSystem")
    assert [spk.get_global("partition_starts", t) for t in range(P)] == list(O.array("partition_starts"))
    assert rel_err(x, O.solve(b)) <= TOL
    assert rel_err(x, x_true) <= TOL


def test_legacy_single_call_and_device_pointers():
    import torch
    L = synth.banded_lower(50000, seed=4)
    x_true, b = synth.make_rhs(L, seed=4)
    x = np.zeros(L.m)
    spk.spike_pstrsv("L", L.m, L.a, L.ia, L.ja, b.copy(), x, 8)
    assert rel_err(x, x_true) <= TOL
    dev = torch.device("cuda:0")
    da = torch.from_numpy(L.a).to(dev)
    dia = torch.from_numpy(L.ia).to(dev)
    dja = torch.from_numpy(L.ja).to(dev)
    db = torch.from_numpy(b).to(dev)
    dx = torch.zeros(L.m, dtype=torch.float64, device=dev)
    spk.spike_pstrsv_preproc(da, dia, dja, L.m, 8, "L")
    spk.spike_pstrsv_solve("L", L.m, db, dx, 8)
    torch.cuda.synchronize()
    assert rel_err(dx.cpu().numpy(), x) <= TOL
    S = spk.System().preproc(da, dia, dja, L.m, 8, "L")
    dx2 = torch.zeros_like(dx)
    S.solve_device(db.data_ptr(), dx2.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert rel_err(dx2.cpu().numpy(), x) <= TOL


def test_timed_variants_fill_timers():
    L = synth.banded_lower(20000, seed=1)
    _, b = synth.make_rhs(L)
    x = np.zeros(L.m)
    spk._spike_pstrsv_preproc(L.a, L.ia, L.ja, L.m, 4, "L")
    spk._spike_pstrsv_solve("L", L.m, b, x, 4)
    assert spk.get_global("produceS_timer_pstrsv3") > 0
    assert spk.get_global("computeY_timer", 0) > 0
    assert spk.get_global("solveD2_timer", 0) > 0


def test_clobbered_rhs_matches_reference_semantics():
    U = synth.transpose(synth.banded_lower(5000, seed=6))
    _, b = synth.make_rhs(U, seed=2)
    spk.set_flag("SPK_CLOBBER_B", 1)
    try:
        bb = b.copy()
        x = np.zeros(U.m)
        spk.spike_pstrsv_preproc(U.a, U.ia, U.ja, U.m, 4, "U")
        spk.spike_pstrsv_solve("U", U.m, bb, x, 4)
    finally:
        spk.set_flag("SPK_CLOBBER_B", 0)
    st = spk.legacy_structure()
    n = U.m
    ID, JD, D = st["ID"], st["JD"], st["D"]
    want = b.copy()
    for r in range(n):
        lo, hi = ID[n + r], ID[n + r + 1]
        if hi > lo:
            want[r] = b[r] - float(np.dot(D[lo:hi], x[JD[lo:hi]]))
    assert rel_err(bb, want) <= TOL


def _drop_entries(A, drop):
    keep = np.ones(A.nnz, bool)
    keep[list(drop)] = False
    rows = np.repeat(np.arange(A.m), np.diff(A.ia))[keep]
    ia = np.zeros(A.m + 1, np.int32)
    np.cumsum(np.bincount(rows, minlength=A.m), out=ia[1:])
    return synth.CSR(A.m, ia, A.ja[keep].copy(), A.a[keep].copy())


def test_errors_are_reported_not_crashes():
    L = synth.poisson2d_lower(4)  # 16 rows
    with pytest.raises(spk.SpkError) as e:
        spk.System().preproc(L.a, L.ia, L.ja, L.m, L.m + 1, "L")
    assert e.value.code == -1
    with pytest.raises(spk.SpkError) as e:
        spk.System().preproc(L.a, L.ia, L.ja, L.m, 2, "Q")
    assert e.value.code == -1
    bad = synth.CSR(L.m, L.ia.copy(), L.ja.copy(), L.a.copy())
    q = L.ia[5]
    bad.ja[q], bad.ja[q + 1] = L.ja[q + 1], L.ja[q]  # unsorted row 5
    with pytest.raises(spk.SpkError) as e:
        spk.System().preproc(bad.a, bad.ia, bad.ja, bad.m, 2, "L")
    assert e.value.code == -2 and "row 5" in str(e.value)
    U = synth.transpose(L)
    nodiag = _drop_entries(U, [U.ia[3]])  # row 3 loses its diagonal
    with pytest.raises(spk.SpkError) as e:
        spk.System().preproc(nodiag.a, nodiag.ia, nodiag.ja, nodiag.m, 2, "U")
    assert e.value.code == -2 and "row 3" in str(e.value)
    empty = _drop_entries(U, range(U.ia[7], U.ia[8]))  # row 7 empty
    with pytest.raises(spk.SpkError) as e:
        spk.System().preproc(empty.a, empty.ia, empty.ja, empty.m, 2, "U")
    assert e.value.code == -2 and "row 7" in str(e.value)
    # a solve that does not match the preprocessed system is reported; x untouched
    spk.spike_pstrsv_preproc(L.a, L.ia, L.ja, L.m, 2, "L")
    x = np.full(L.m, 7.0)
    spk.spike_pstrsv_solve("L", L.m, np.ones(L.m), x, 3)
    assert np.all(x == 7.0)
    assert spk.last_error()[0] == -5


_BANDED = {}
X_SAMPLES = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "full_x_samples.npz")


def banded_full(uplo):
    if uplo not in _BANDED:
        _BANDED.clear()  # one full-size matrix at a time (host memory)
        L = synth.banded_lower(4194304, seed=0)
        _BANDED[uplo] = L if uplo == "L" else synth.transpose(L)
    return _BANDED[uplo]


def x_sample_index(m):
    idx = np.concatenate([np.arange(0, m, 997), np.arange(64), np.arange(m - 64, m)])
    return np.unique(idx)


@pytest.mark.parametrize("uplo,P", [(u, P) for u in "LU" for P in (16, 64, 256, 1024)])
def test_full_size_banded(uplo, P):
    """The full banded workload (m = 4,194,304) at every swept partition count:
    every structure array bit-exact against the reference's digests, x within
    1e-12 of the reference's x (at the sampled rows), of the sequential
    substitution and of x_true."""
    A = banded_full(uplo)
    x_true, b = synth.make_rhs(A, seed=0)
    S = gpu_system(A, P, uplo, 1)
    x = S.solve(b)
    xs = oracle.sequential_solve(A, b, uplo)
    assert rel_err(x, xs) <= TOL
    assert rel_err(x, x_true) <= TOL
    key = f"banded4194304_{uplo}_P{P}"
    rec = DIGEST[key]
    got = trim_S(S.structure(), rec["sizes"]["S"])
    bad = [k for k, h in rec["arrays"].items() if sha(got[k]) != h]
    bad += [k for k, v in rec["scalars"].items() if int(got[k]) != v]
    assert bad == []
    xr = np.load(X_SAMPLES)[key]
    xi = x[x_sample_index(A.m)]
    assert np.linalg.norm(xi - xr) <= TOL * np.linalg.norm(xr)
    assert abs(np.linalg.norm(x) - rec["x_ref_norm"]) <= TOL * rec["x_ref_norm"]


@pytest.mark.parametrize("path", SMALL[:6], ids=[os.path.basename(p)[6:-4] for p in SMALL[:6]])
def test_gpu_exact_mode_matches_golden(path):
    A, P, flb, uplo, b, x_ref, want = load_small(path)
    S = gpu_system(A, P, uplo, flb).set_truncation(-1.0)
    assert S.scalar("rows_phase4") >= 0
    assert rel_err(S.solve(b), x_ref) <= TOL


def test_truncation_engages_on_decaying_spikes_and_stays_accurate():
    L = synth.banded_lower(262144, seed=9)
    x_true, b = synth.make_rhs(L, seed=9)
    xs = oracle.sequential_solve(L, b, "L")
    S = gpu_system(L, 64, "L", 1)
    assert S.scalar("rows_phase4") < L.m // 2      # D2 work cut to the coupled rows
    assert S.scalar("kept_reduced_rows") == 0       # every reduced row below 2^-60
    x = S.solve(b)
    assert rel_err(x, xs) <= TOL
    E = gpu_system(L, 64, "L", 1).set_truncation(-1.0)
    assert E.scalar("rows_phase4") > L.m // 2
    xe = E.solve(b)
    assert rel_err(xe, xs) <= TOL
    assert rel_err(x, xe) <= 1e-15


def test_csr_fallback_solver_matches_oracle(monkeypatch):
    """The CSR segment solver (used when the sliced-ELL layout would pad too much)."""
    monkeypatch.setenv("SPK_DISABLE_ELL", "1")
    for name, A, P in random_cases(12):
        O = oracle.Oracle()
        O.preproc(A, P, uplo="U", flb=1)
        S = gpu_system(A, P, "U", 1)
        assert S.scalar("ell") == 0
        _, b = synth.make_rhs(A, seed=1)
        assert rel_err(S.solve(b), O.solve(b)) <= TOL, name
    L = synth.banded_lower(100000, seed=3)
    x_true, b = synth.make_rhs(L, seed=3)
    S = gpu_system(L, 64, "L", 1)
    assert rel_err(S.solve(b), x_true) <= TOL


def test_ell_layout_is_used_for_banded():
    L = synth.banded_lower(10000, seed=3)
    S = gpu_system(L, 8, "L", 1)
    assert S.scalar("ell") == 1
    U = synth.mirror(L)
    offd = np.diff(U.ia) - 1
    widths = [int(offd[j:j + 32].max()) for j in range(0, U.m, 32)]
    assert S.scalar("ell_entries") == 32 * sum(widths)
