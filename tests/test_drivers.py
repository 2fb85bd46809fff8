"""The reference's own drivers (test/runtime_analysis.c, example_usage.c),
compiled from the reference tree against libspike_pstrsv_b200.so and
libspike_pstrsv_mklcompat.so (include/compat headers): they link, load and
print their usage text without a GPU.  Their GPU runs are in
test_gpu_drivers.py."""
import os
import subprocess

import pytest

import oracle

DRIVERS = [oracle.PROFILER_BIN, oracle.EXAMPLE_BIN]


@pytest.mark.parametrize("path", DRIVERS, ids=os.path.basename)
def test_driver_links_and_prints_usage(path):
    if not os.path.exists(path):
        pytest.skip(f"{path} not built (make -C oracle drivers, with the reference tree present)")
    out = subprocess.run([path], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stderr
    assert out.stdout.startswith("Usage:")


def test_every_compat_symbol_is_exported():
    """Every function include/compat/mkl.h declares is exported by
    libspike_pstrsv_mklcompat.so (the MKL entry points the reference's drivers call)."""
    import re

    from conftest import ROOT
    from spike_pstrsv_b200 import build

    text = open(os.path.join(ROOT, "include", "compat", "mkl.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    funcs = set(re.findall(r"^\s*(?:const\s+)?[a-z_]+\s*\**\s*([A-Za-z_][A-Za-z0-9_]*)\s*\(", text, flags=re.M))
    assert {"mkl_cspblas_dcsrtrsv", "mkl_sparse_d_trsv", "mkl_sparse_d_create_csr", "mkl_dcsrmv",
            "cblas_dcopy", "mkl_malloc", "mkl_free"} <= funcs
    lib = build.build_compat()
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True, check=True)
    exported = {line.split()[-1] for line in out.stdout.splitlines() if line.strip()}
    assert sorted(funcs - exported) == []
