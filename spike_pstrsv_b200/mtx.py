"""MatrixMarket ingest through the library's reader (spk_mtx_read, the C
restatement of the reference's matrixMarketToCSR, src/misc.c:109-245).  Host
code only: works without a GPU."""
from __future__ import annotations

import ctypes

import numpy as np

from .capi import SpkError, lib
from .synth import CSR


def read(path: str, uplo: str = "N", symm: str = "N") -> CSR:
    """CSR of the file: uplo 'U' / 'L' keeps that triangle (diagonal included),
    'N' everything; symm 'Y' mirrors the off-diagonal entries of a symmetric file."""
    L = lib()
    dp, ip = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
    L.spk_mtx_read.argtypes = [ctypes.c_char_p, ctypes.c_char, ctypes.c_char, ctypes.POINTER(dp),
                               ctypes.POINTER(ip), ctypes.POINTER(ip), ctypes.POINTER(ctypes.c_int),
                               ctypes.POINTER(ctypes.c_int)]
    L.spk_mtx_free.argtypes = [dp, ip, ip]
    a, ia, ja = dp(), ip(), ip()
    n, nnz = ctypes.c_int(), ctypes.c_int()
    rc = L.spk_mtx_read(str(path).encode(), uplo.encode(), symm.encode(), ctypes.byref(a), ctypes.byref(ia),
                        ctypes.byref(ja), ctypes.byref(n), ctypes.byref(nnz))
    if rc != 0:
        raise SpkError(rc, L.spk_last_error().decode())
    try:
        A = CSR(n.value, np.ctypeslib.as_array(ia, (n.value + 1,)).copy(),
                np.ctypeslib.as_array(ja, (max(nnz.value, 1),))[: nnz.value].copy(),
                np.ctypeslib.as_array(a, (max(nnz.value, 1),))[: nnz.value].copy())
    finally:
        L.spk_mtx_free(a, ia, ja)
    return A


def write(path: str, A: CSR, comment: str = "") -> None:
    """Coordinate real general file of A (1-based)."""
    rows = np.repeat(np.arange(A.m), np.diff(A.ia.astype(np.int64)))
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n")
        if comment:
            f.write(f"% {comment}\n")
        f.write(f"{A.m} {A.m} {A.nnz}\n")
        for r, c, v in zip(rows, A.ja, A.a):
            f.write(f"{int(r) + 1} {int(c) + 1} {float(v)!r}\n")
