"""MatrixMarket ingest (matrixMarketToCSR / spk_mtx_read) against the reference's
own reader built from its sources (oracle/_ref), against CSR built here, and its
error paths.  Host code: runs without a GPU."""
import ctypes

import numpy as np
import pytest

import oracle
from spike_pstrsv_b200 import capi, mtx, synth

GENERAL = """%%MatrixMarket matrix coordinate real general
% a comment line
%
5 5 10
3 3 3.0
1 1 1.0
2 1 -0.5
5 5 5.0
2 2 2.0
4 4 4.0
5 3 0.25
3 1 0.125
4 2 -2.0
1 4 9.0
"""

SYMMETRIC = """%%MatrixMarket matrix coordinate real symmetric
4 4 7
1 1 4.0
2 2 4.0
3 3 4.0
4 4 4.0
2 1 -1.0
3 2 -1.0
4 3 -1.0
"""


def _dense(A):
    D = np.zeros((A.m, A.m))
    for r in range(A.m):
        for q in range(A.ia[r], A.ia[r + 1]):
            D[r, A.ja[q]] += A.a[q]
    return D


def _reference_read(path, uplo, symm):
    if not oracle.Reference.available():
        pytest.skip(oracle.Reference.missing_reason())
    L = oracle.Reference.lib()
    dp, ip = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
    f = L.matrixMarketToCSR
    f.argtypes = [ctypes.c_char_p, ctypes.POINTER(dp), ctypes.POINTER(ip), ctypes.POINTER(ip),
                  ctypes.POINTER(ctypes.c_int), ctypes.c_char, ctypes.c_char]
    a, ia, ja, n = dp(), ip(), ip(), ctypes.c_int()
    f(str(path).encode(), ctypes.byref(a), ctypes.byref(ia), ctypes.byref(ja), ctypes.byref(n), uplo.encode(),
      symm.encode())
    m = n.value
    iah = np.ctypeslib.as_array(ia, (m + 1,)).copy()
    nnz = int(iah[-1])
    return synth.CSR(m, iah, np.ctypeslib.as_array(ja, (nnz,)).copy(), np.ctypeslib.as_array(a, (nnz,)).copy())


@pytest.mark.parametrize("uplo", ["N", "L", "U"])
def test_general_file_matches_the_reference_reader(tmp_path, uplo):
    p = tmp_path / "g.mtx"
    p.write_text(GENERAL)
    A = mtx.read(p, uplo, "N")
    R = _reference_read(p, uplo, "N")
    assert A.m == R.m == 5
    assert np.array_equal(A.ia, R.ia) and np.array_equal(A.ja, R.ja) and np.array_equal(A.a, R.a)
    full = np.zeros((5, 5))
    for line in GENERAL.splitlines()[4:]:
        r, c, v = line.split()
        full[int(r) - 1, int(c) - 1] = float(v)
    want = {"N": full, "L": np.tril(full), "U": np.triu(full)}[uplo]
    assert np.array_equal(_dense(A), want)


@pytest.mark.parametrize("uplo", ["L", "U", "N"])
def test_symmetric_file_is_mirrored(tmp_path, uplo):
    p = tmp_path / "s.mtx"
    p.write_text(SYMMETRIC)
    A = mtx.read(p, uplo, "Y")
    R = _reference_read(p, uplo, "Y")
    assert np.array_equal(A.ia, R.ia) and np.array_equal(A.ja, R.ja) and np.array_equal(A.a, R.a)
    T = 4.0 * np.eye(4) - np.eye(4, k=1) - np.eye(4, k=-1)
    want = {"N": T, "L": np.tril(T), "U": np.triu(T)}[uplo]
    assert np.array_equal(_dense(A), want)


def test_round_trip_of_a_banded_system(tmp_path):
    L = synth.banded_lower(3000, seed=4)
    p = tmp_path / "b.mtx"
    mtx.write(p, L, comment="banded")
    A = mtx.read(p, "L", "N")
    assert np.array_equal(A.ia, L.ia) and np.array_equal(A.ja, L.ja) and np.array_equal(A.a, L.a)
    R = _reference_read(p, "L", "N")
    assert np.array_equal(R.ia, L.ia) and np.array_equal(R.ja, L.ja) and np.array_equal(R.a, L.a)


def test_empty_rows_keep_their_row_pointers(tmp_path):
    """Row 2 has no entry in the upper triangle: its pointer repeats (the reference
    advances one pointer per row change and shifts the rows after it)."""
    p = tmp_path / "e.mtx"
    p.write_text("%%MatrixMarket matrix coordinate real general\n3 3 3\n1 1 1.0\n3 3 3.0\n2 1 5.0\n")
    A = mtx.read(p, "U", "N")
    assert list(A.ia) == [0, 1, 1, 2]
    assert list(A.ja) == [0, 2] and list(A.a) == [1.0, 3.0]


@pytest.mark.parametrize("text", [
    "%%MatrixMarket matrix coordinate pattern general\n2 2 1\n1 1\n",   # no values
    "%%MatrixMarket matrix coordinate real general\n2 2 2\n1 1 1.0\n",  # missing entry
    "%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 1.0\n",  # out of range
    "%%MatrixMarket matrix coordinate real general\n",                  # no size line
])
def test_bad_files_are_errors(tmp_path, text):
    p = tmp_path / "bad.mtx"
    p.write_text(text)
    with pytest.raises(capi.SpkError):
        mtx.read(p)


def test_missing_file_and_bad_flags():
    with pytest.raises(capi.SpkError):
        mtx.read("/nonexistent/file.mtx")
    with pytest.raises(capi.SpkError):
        mtx.read(__file__, "X", "N")
