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
# MKL entry points for the reference's drivers (include/compat/mkl.h), apart from
# the solver library so that a process with the real MKL never sees them twice.
COMPAT_LIB = os.path.join(HERE, "libspike_pstrsv_mklcompat.so")
COMPAT_SRC = "mklcompat.cu"

SOURCES = ["preproc.cu", "solve.cu", "chain.cu", "capi.cu", "server.cu", "mtx.cu", "reorder.cu"]
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


def build_compat(force: bool = False, verbose: bool = False) -> str:
    """libspike_pstrsv_mklcompat.so: host MKL helpers and cuSPARSE SpSV comparators."""
    src = os.path.join(CSRC, COMPAT_SRC)
    hdr = os.path.join(ROOT, "include", "compat", "mkl.h")
    if not force and os.path.exists(COMPAT_LIB) and all(
            os.path.getmtime(d) <= os.path.getmtime(COMPAT_LIB) for d in (src, hdr)):
        return COMPAT_LIB
    tmp = COMPAT_LIB + ".tmp"
    cmd = [nvcc()] + ARCH + FLAGS[:-2] + ["-Xcompiler", "-fopenmp", "-o", tmp, src, "-lcusparse", "-lgomp"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(tmp, COMPAT_LIB)
    return COMPAT_LIB


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every source to its own object in parallel (no device code crosses
    files, so separate compilation gives the same kernels), then link one .so;
    then the MKL compatibility library."""
    build_compat(force, verbose)
    if not force and up_to_date():
        return LIB
    from concurrent.futures import ThreadPoolExecutor

    tmp = LIB + ".tmp"
    extra = os.environ.get("SPK_NVCC_EXTRA", "").split()  # e.g. -DSPK_DEVICE_CHECKS (checked build)
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    compile_flags = [f for f in FLAGS if f != "-shared"]
    inc = ["-I" + os.path.join(ROOT, "include")]

    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(ROOT, "include", "spike_pstrsv.h"))
    stamp = os.path.join(objdir, "flags.txt")
    flags_line = " ".join(ARCH + compile_flags + extra)
    same_flags = os.path.exists(stamp) and open(stamp).read() == flags_line

    def compile_one(src: str) -> str:
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        if (not force and same_flags and os.path.exists(obj)
                and all(os.path.getmtime(d) <= os.path.getmtime(obj) for d in [src] + headers)):
            return obj
        cmd = [nvcc()] + ARCH + compile_flags + extra + inc + ["-c", "-o", obj, src]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        return obj

    with ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 1)) as pool:
        objs = list(pool.map(compile_one, sources()))
    with open(stamp, "w") as f:
        f.write(flags_line)
    subprocess.run([nvcc()] + ARCH + ["-shared", "-o", tmp] + objs, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
