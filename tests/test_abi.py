"""C-ABI library: builds, loads without a GPU, exports every symbol the public
header declares, and refuses to compute without a CUDA device (no CPU fallback)."""
import os
import re
import subprocess

import pytest

from conftest import HAS_CUDA, ROOT
from spike_pstrsv_b200 import build, capi

HEADER = os.path.join(ROOT, "include", "spike_pstrsv.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    funcs = set(re.findall(r"^\s*(?:const\s+)?[a-z_]+\s*\**\s*\**([A-Za-z_][A-Za-z0-9_]*)\s*\(", text, flags=re.M))
    funcs -= {"if", "return"}
    vars_ = set(re.findall(r"^\s*extern\s+[A-Za-z_ ]+?\s\**([A-Za-z_][A-Za-z0-9_]*)\s*(?:\[|;)", text, flags=re.M))
    return funcs, vars_


def exported():
    out = subprocess.run(["nm", "-D", "--defined-only", build.LIB], capture_output=True, text=True, check=True)
    return {line.split()[-1] for line in out.stdout.splitlines() if line.strip()}


def test_library_builds_and_loads():
    assert os.path.exists(build.build())
    capi.lib()


def test_every_declared_symbol_is_exported():
    funcs, vars_ = declared_symbols()
    assert {"spike_pstrsv_preproc", "_spike_pstrsv_preproc", "spike_pstrsv", "spike_pstrsv_solve",
            "_spike_pstrsv_solve", "free_PSTRSV3", "logPSTRSV3"} <= funcs
    assert {"PSTRSV_VERBOSE", "FORCE_LOAD_BALANCE", "IS_MATRIX_PARTITIONED", "numRowsReducedSystem",
            "computeY_timer", "partition_starts"} <= vars_
    missing = sorted((funcs | vars_) - exported())
    assert missing == []


def test_reference_flag_defaults():
    assert capi.get_flag("FORCE_LOAD_BALANCE") == 1
    assert capi.get_flag("PSTRSV_VERBOSE") == 0
    assert capi.get_flag("IS_MATRIX_PARTITIONED") == 0


@pytest.mark.skipif(HAS_CUDA, reason="checks the no-GPU behaviour")
def test_no_cpu_fallback_without_gpu():
    with pytest.raises(capi.SpkError):
        capi.System()


def build_c_driver(tmp_path):
    exe = str(tmp_path / "example_driver")
    src = os.path.join(ROOT, "tests", "c", "example_driver.c")
    libdir = os.path.dirname(build.LIB)
    subprocess.run(["/usr/bin/gcc", "-O2", "-o", exe, src, "-I" + os.path.join(ROOT, "include"),
                    "-L" + libdir, "-lspike_pstrsv_b200", "-Wl,-rpath," + libdir, "-lm"], check=True)
    return exe


def test_c_caller_compiles_and_links(tmp_path):
    """A C program in the reference's example_usage.c call pattern builds against
    include/spike_pstrsv.h and links libspike_pstrsv_b200.so."""
    assert os.path.exists(build_c_driver(tmp_path))


@pytest.mark.gpu
def test_c_caller_runs(tmp_path):
    exe = build_c_driver(tmp_path)
    out = subprocess.run([exe, "96", "6"], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "Reduced system size" in out.stdout  # logPSTRSV3 text format


@pytest.mark.gpu
def test_c_caller_runs_on_a_matrix_market_file(tmp_path):
    """The profiler's way in: matrixMarketToCSR then the drop-in solve."""
    from spike_pstrsv_b200 import mtx, synth
    L = synth.poisson2d_lower(64)
    path = str(tmp_path / "poisson64.mtx")
    mtx.write(path, L)
    exe = build_c_driver(tmp_path)
    out = subprocess.run([exe, "64", "4", path], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert f"read {path}: {L.m} rows, {L.nnz} entries" in out.stdout
