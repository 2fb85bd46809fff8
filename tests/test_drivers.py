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
