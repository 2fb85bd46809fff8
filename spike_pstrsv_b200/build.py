"""Build the sm_100a library libspike_pstrsv_b200.so in-tree with nvcc.

The library is plain C ABI (include/spike_pstrsv.h); nothing here depends on
PyTorch.  nvcc cross-compiles, so this runs on machines without a GPU.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libspike_pstrsv_b200.so")

SOURCES = ["preproc.cu", "solve.cu", "chain.cu", "capi.cu", "server.cu", "mtx.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC,-O2",
         "-Xptxas", "-warn-spills"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return [os.path.join(CSRC, f) for f in SOURCES]


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    deps = sources() + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    deps.append(os.path.join(ROOT, "include", "spike_pstrsv.h"))
    return all(os.path.getmtime(d) <= t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    tmp = LIB + ".tmp"
    extra = os.environ.get("SPK_NVCC_EXTRA", "").split()  # e.g. -DSPK_DEVICE_CHECKS (checked build)
    cmd = [nvcc()] + ARCH + FLAGS + extra + ["-I" + os.path.join(ROOT, "include"), "-o", tmp] + sources()
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
