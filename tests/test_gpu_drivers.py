"""The reference's profiler (test/runtime_analysis.c) and example
(example_usage.c), unmodified, built against this library with the MKL
comparators answered by cuSPARSE SpSV (include/compat/mkl.h), run on a
MatrixMarket file: every solver's 2-norm error stays under the reference's own
1e-4 acceptance threshold (no "!!!" line), the runtime analysis is printed, and
the METIS path runs the library's matrixReordering."""
import os
import re
import subprocess

import numpy as np
import pytest
import scipy.sparse as sp

import oracle

pytestmark = pytest.mark.gpu


def need(path):
    if not os.path.exists(path):
        pytest.skip(f"{path} not built (make -C oracle drivers, with the reference tree present)")


def write_symmetric_mtx(path, k):
    """The 2-D 5-point Laplacian on a k x k grid as a 'symmetric' MatrixMarket
    file (lower triangle stored)."""
    T = sp.diags([-1.0, 4.0, -1.0], [-1, 0, 1], (k, k))
    A = (sp.kron(sp.eye(k), T) + sp.kron(sp.diags([-1.0, -1.0], [-1, 1], (k, k)), sp.eye(k))).tocoo()
    keep = A.row >= A.col
    r, c, v = A.row[keep], A.col[keep], A.data[keep]
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real symmetric\n")
        f.write(f"{k * k} {k * k} {len(v)}\n")
        for i, j, x in zip(r, c, v):
            f.write(f"{i + 1} {j + 1} {x:.17g}\n")


def run(args, timeout=600):
    out = subprocess.run(args, capture_output=True, text=True, timeout=timeout)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    return out.stdout


def runtimes(text):
    rows = re.findall(r"^(.*Triangular Solver)\s*\|\s*Min\. runtime: ([0-9.]+) ms", text, re.M)
    return {name.strip(): float(ms) for name, ms in rows}


@pytest.mark.parametrize("uplo,metis", [("L", "N"), ("U", "N"), ("U", "Y"), ("L", "Y")])
def test_profiler_runs_against_library(tmp_path, uplo, metis):
    need(oracle.PROFILER_BIN)
    mtx = str(tmp_path / "poisson64.mtx")
    write_symmetric_mtx(mtx, 64)
    text = run([oracle.PROFILER_BIN, mtx, "4", uplo, "Y", metis])
    assert "!!!" not in text, text
    assert "Runtime Analysis of spike_pstrsv" in text
    t = runtimes(text)
    assert set(t) == {"MKL Seq. Triangular Solver", "MKL Par. Triangular Solver", "SPARSKIT Triangular Solver",
                      "Parallel Triangular Solver"}, text
    assert all(np.isfinite(v) and v > 0 for v in t.values()), t
    if metis == "Y":
        assert "Matrix reodering is completed." in text


@pytest.mark.parametrize("uplo", ["L", "U"])
def test_example_runs_against_library(tmp_path, uplo):
    need(oracle.EXAMPLE_BIN)
    mtx = str(tmp_path / "poisson48.mtx")
    write_symmetric_mtx(mtx, 48)
    text = run([oracle.EXAMPLE_BIN, mtx, "4", uplo, "Y"])
    m = re.search(r"spike_pstrsv residual: ([0-9.eE+-]+)", text)
    assert m, text
    assert float(m.group(1)) <= 1e-4
