"""The CPU oracle (oracle/spike_oracle.c) against the reference: golden fixtures
made by the reference's own sources (tests/golden/make_golden.py) and, where the
reference checker library is present, live bit-exact comparisons."""
import glob
import hashlib
import json
import os

import numpy as np
import pytest

import oracle
from cases import random_cases, rel_err, struct_diff
from spike_pstrsv_b200 import synth

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def load_small(path):
    z = np.load(path)
    m, P, flb, up = (int(v) for v in z["meta"])
    A = synth.CSR(m, z["ia"], z["ja"], z["a"])
    st = {k[2:]: z[k] for k in z.files if k.startswith("s_")}
    st.update({k[2:]: int(z[k]) for k in z.files if k.startswith("c_")})
    return A, P, flb, chr(up), z["b"], z["x_ref"], st


def trim_S(st: dict, n: int) -> dict:
    """The reference's S has ends_S[P-1] elements; the restatement pads to totalArea."""
    out = dict(st)
    S = np.asarray(st["S"])
    assert not S[n:].any()
    out["S"] = S[:n]
    return out


SMALL = sorted(glob.glob(os.path.join(GOLDEN, "small_*.npz")))


@pytest.mark.parametrize("path", SMALL, ids=[os.path.basename(p)[6:-4] for p in SMALL])
def test_oracle_matches_golden_small(path):
    A, P, flb, uplo, b, x_ref, want = load_small(path)
    O = oracle.Oracle()
    assert O.preproc(A, P, uplo=uplo, flb=flb) == 0
    got = trim_S(O.structure(), len(want["S"]))
    assert struct_diff(got, want) == []
    assert rel_err(O.solve(b), x_ref) <= 1e-12


def digest_cases():
    with open(os.path.join(GOLDEN, "digest.json")) as f:
        return json.load(f)


def make_case(rec):
    gen = rec["gen"]
    if gen == "poisson128":
        L = synth.poisson2d_lower(128)
    elif gen == "banded65536":
        L = synth.banded_lower(65536, seed=0)
    elif gen == "banded4194304":
        L = synth.banded_lower(4194304, seed=0)
    else:
        raise KeyError(gen)
    return L if rec["uplo"] == "L" else synth.transpose(L)


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


DIGEST = digest_cases()
DIGEST_SMALL = {k: v for k, v in DIGEST.items() if v["m"] <= 65536}


@pytest.mark.parametrize("name", sorted(DIGEST_SMALL))
def test_oracle_matches_golden_digest(name):
    rec = DIGEST[name]
    A = make_case(rec)
    O = oracle.Oracle()
    assert O.preproc(A, rec["P"], uplo=rec["uplo"], flb=rec["flb"]) == 0
    got = trim_S(O.structure(), rec["sizes"]["S"])
    bad = [k for k, h in rec["arrays"].items() if sha(got[k]) != h]
    bad += [k for k, v in rec["scalars"].items() if int(got[k]) != v]
    assert bad == []
    x_true, b = synth.make_rhs(A, seed=0)
    x = O.solve(b)
    assert rel_err(x, x_true) <= 1e-12


needs_ref = pytest.mark.skipif(not oracle.Reference.available(), reason=oracle.Reference.missing_reason())


@needs_ref
@pytest.mark.parametrize("flb", [0, 1])
def test_oracle_matches_reference_random(flb):
    failures = []
    for name, A, P in random_cases(40):
        R = oracle.Reference()
        R.preproc(A, P, flb=flb)
        want = R.structure()
        O = oracle.Oracle()
        assert O.preproc(A, P, uplo="U", flb=flb) == 0
        got = trim_S(O.structure(), len(want["S"]))
        bad = struct_diff(got, want)
        x_true, b = synth.make_rhs(A, seed=1)
        if bad or rel_err(O.solve(b), R.solve(b)) > 1e-12:
            failures.append((name, bad))
    assert failures == []


@needs_ref
@pytest.mark.parametrize("P", [2, 7, 33])
def test_oracle_matches_reference_banded_lower(P):
    L = synth.banded_lower(20000, seed=5)
    R = oracle.Reference()
    R.preproc(synth.mirror(L), P, flb=1)
    want = R.structure()
    O = oracle.Oracle()
    assert O.preproc(L, P, uplo="L", flb=1) == 0
    got = trim_S(O.structure(), len(want["S"]))
    assert struct_diff(got, want) == []


def test_sequential_oracle_against_scipy():
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl
    L = synth.banded_lower(3000, seed=2)
    x_true, b = synth.make_rhs(L, seed=3)
    M = sp.csr_matrix((L.a, L.ja, L.ia), shape=(L.m, L.m))
    xl = oracle.sequential_solve(L, b, "L")
    assert rel_err(xl, spl.spsolve_triangular(M, b, lower=True)) <= 1e-13
    U = synth.transpose(L)
    _, bu = synth.make_rhs(U, seed=3)
    xu = oracle.sequential_solve(U, bu, "U")
    assert rel_err(xu, x_true) <= 1e-13


def test_mirror_is_involution_and_upper():
    L = synth.poisson2d_lower(16)
    U = synth.mirror(L)
    assert all(U.ja[U.ia[r]] == r for r in range(U.m))
    back = synth.mirror(U)
    assert np.array_equal(back.ia, L.ia) and np.array_equal(back.ja, L.ja) and np.array_equal(back.a, L.a)


def test_oracle_rejects_more_partitions_than_rows():
    L = synth.poisson2d_lower(2)
    O = oracle.Oracle()
    assert O.preproc(L, 5, uplo="L") < 0
