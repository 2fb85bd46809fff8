"""ORACLE -- test infrastructure only.

CPU checkers for the spike_pstrsv hot path.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg import this
package, and only to check or time against the CUDA path; the product never
routes through it.

* ``Oracle``    -- ctypes wrapper of ``liboracle.so``, the sequential C
  restatement of the reference algorithm (``spike_oracle.c``).
* ``Reference`` -- ctypes wrapper of ``_ref/libspike_ref.so``, the reference's
  own sources compiled with the MKL shim (``Makefile`` target ``ref``).  Present
  only where the reference tree was available at build time.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libspike_ref.so")
# The reference's own drivers built against the GPU library (Makefile target
# ``drivers``); they exercise the product, the tests only run them.
PROFILER_BIN = os.path.join(HERE, "_ref", "runtimeAnalysis")
EXAMPLE_BIN = os.path.join(HERE, "_ref", "exampleUsage")

_DT = {"d": np.float64, "i": np.int32, "q": np.int64, "c": np.int8}
_CT = {"d": ctypes.c_double, "i": ctypes.c_int32, "q": ctypes.c_int64, "c": ctypes.c_int8}

STRUCT_ARRAYS = [
    "partition_starts", "partition_ends", "partition_numRows",
    "D", "ID", "JD", "starts_D", "ends_D", "starts_R", "ends_R",
    "hasDependences", "hasReflections", "hasToCalculateSs", "isOptimizeds",
    "numRows_S", "numCols_S", "starts_S", "ends_S", "start_intervals", "end_intervals",
    "T2", "IT2", "JT2", "starts_D0", "ends_D0", "starts_D1", "ends_D1", "starts_D2", "ends_D2",
    "mapR", "starts_mapR", "ends_mapR", "S", "mapReducedX", "T", "IT", "JT",
]
STRUCT_SCALARS = ["numRowsReducedSystem", "numNnzsReducedSystem", "reducedSystemSolverStart",
                  "isReducedSystemNecessary"]


def build(ref: bool | None = None) -> None:
    """Compile liboracle.so (and the reference checker when its sources exist)."""
    import subprocess

    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
    src = ref_source_dir()
    if ref is None:
        ref = os.path.isdir(src)
    if ref:
        subprocess.run(["make", "-s", "-C", HERE, "ref", "SPK_REF_SRC=" + src], check=True)
        # the reference's profiler and example, linked against the GPU library
        # (built before this by __graft_entry__.build)
        subprocess.run(["make", "-s", "-C", HERE, "drivers", "SPK_REF_SRC=" + src], check=True)


def ref_source_dir() -> str:
    """The reference tree's ``src/`` folder: ``$SPK_REF_SRC`` when set, else a
    checkout named ``reference`` beside the repository (the Makefile's default)."""
    env = os.environ.get("SPK_REF_SRC")
    if env:
        return os.path.abspath(env)
    return os.path.abspath(os.path.join(HERE, "..", "..", "reference", "src"))


def _i32(x):
    return np.ascontiguousarray(x, dtype=np.int32)


def _f64(x):
    return np.ascontiguousarray(x, dtype=np.float64)


class Oracle:
    """Sequential C restatement of the reference (one preprocessed matrix per object)."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            lib = ctypes.CDLL(ORACLE_SO)
            lib.spko_create.restype = ctypes.c_void_p
            lib.spko_destroy.argtypes = [ctypes.c_void_p]
            lib.spko_preproc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_char, ctypes.c_int, ctypes.c_void_p,
                                         ctypes.c_void_p]
            lib.spko_solve.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
            lib.spko_array.restype = ctypes.c_void_p
            lib.spko_array.argtypes = [ctypes.c_void_p, ctypes.c_char_p,
                                       ctypes.POINTER(ctypes.c_longlong), ctypes.c_char_p]
            lib.spko_scalar.restype = ctypes.c_longlong
            lib.spko_scalar.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
            for f in (lib.spko_udsol, lib.spko_ldsol):
                f.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                              ctypes.c_void_p, ctypes.c_void_p]
            cls._lib = lib
        return cls._lib

    def __init__(self):
        self.h = self.lib().spko_create()

    def __del__(self):
        try:
            self.lib().spko_destroy(self.h)
        except Exception:
            pass

    def preproc(self, A, P: int, uplo: str = "U", flb: int = 1, starts=None, ends=None) -> int:
        self._keep = (_f64(A.a), _i32(A.ia), _i32(A.ja))
        a, ia, ja = self._keep
        st = _i32(starts) if starts is not None else None
        en = _i32(ends) if ends is not None else None
        rc = self.lib().spko_preproc(self.h, a.ctypes.data, ia.ctypes.data, ja.ctypes.data,
                                     int(A.m), int(P), uplo.encode()[:1], int(flb),
                                     st.ctypes.data if st is not None else None,
                                     en.ctypes.data if en is not None else None)
        self.m = A.m
        return rc

    def solve(self, b: np.ndarray) -> np.ndarray:
        b = _f64(b)
        x = np.zeros(self.m)
        rc = self.lib().spko_solve(self.h, b.ctypes.data, x.ctypes.data)
        if rc:
            raise RuntimeError(f"oracle solve failed: {rc}")
        return x

    def array(self, name: str) -> np.ndarray:
        cnt = ctypes.c_longlong()
        ty = ctypes.create_string_buffer(2)
        p = self.lib().spko_array(self.h, name.encode(), ctypes.byref(cnt), ty)
        if not p and cnt.value:
            raise KeyError(name)
        t = ty.value.decode() or "i"
        if cnt.value == 0:
            return np.zeros(0, dtype=_DT[t])
        buf = (_CT[t] * cnt.value).from_address(p)
        return np.ctypeslib.as_array(buf).copy()

    def scalar(self, name: str) -> int:
        return int(self.lib().spko_scalar(self.h, name.encode()))

    def structure(self) -> dict:
        out = {k: self.array(k) for k in STRUCT_ARRAYS}
        out.update({k: self.scalar(k) for k in STRUCT_SCALARS})
        return out


def sequential_solve(A, b: np.ndarray, uplo: str) -> np.ndarray:
    """Plain FP64 substitution over the whole matrix (runtime_analysis.c:37-65)."""
    lib = Oracle.lib()
    a, ia, ja, b = _f64(A.a), _i32(A.ia), _i32(A.ja), _f64(b)
    x = np.zeros(A.m)
    f = lib.spko_udsol if uplo.upper() == "U" else lib.spko_ldsol
    f(int(A.m), a.ctypes.data, ia.ctypes.data, ja.ctypes.data, b.ctypes.data, x.ctypes.data)
    return x


class Reference:
    """The reference's own sources (oracle/_ref/libspike_ref.so), driven through its C API.

    Holds process-global state (the reference is single-instance).  Only the
    'U' path is implemented by the reference; 'L' is run through the mirror by
    the caller."""

    _lib = None

    @classmethod
    def available(cls) -> bool:
        return os.path.exists(REF_SO)

    @classmethod
    def missing_reason(cls) -> str:
        return (f"reference checker {REF_SO} not built (make -C oracle ref, with the reference "
                f"sources at {ref_source_dir()} or SPK_REF_SRC)")

    @classmethod
    def lib(cls):
        if cls._lib is None:
            lib = ctypes.CDLL(REF_SO)
            lib.spike_pstrsv_preproc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                 ctypes.c_int, ctypes.c_int, ctypes.c_char]
            lib._spike_pstrsv_preproc.argtypes = lib.spike_pstrsv_preproc.argtypes
            lib.spike_pstrsv_solve.argtypes = [ctypes.c_char, ctypes.c_int, ctypes.c_void_p,
                                               ctypes.c_void_p, ctypes.c_int]
            lib._spike_pstrsv_solve.argtypes = lib.spike_pstrsv_solve.argtypes
            cls._lib = lib
        return cls._lib

    def _sym(self, name, ctype):
        return ctype.in_dll(self.lib(), name)

    def set_flag(self, name: str, value: int) -> None:
        self._sym(name, ctypes.c_int8).value = int(value)

    def preproc(self, A, P: int, flb: int = 1, timed: bool = False) -> None:
        self._keep = (_f64(A.a), _i32(A.ia), _i32(A.ja))
        a, ia, ja = self._keep
        self.set_flag("FORCE_LOAD_BALANCE", flb)
        self.m, self.P = int(A.m), int(P)
        f = self.lib()._spike_pstrsv_preproc if timed else self.lib().spike_pstrsv_preproc
        f(a.ctypes.data, ia.ctypes.data, ja.ctypes.data, self.m, self.P, b"U")

    def solve(self, b: np.ndarray, timed: bool = False) -> np.ndarray:
        """x for one right-hand side; b is copied first (the reference clobbers it).
        Buffers carry a 16-element guard in front: the reference may write x[-1]
        of a segment when a D1 range is empty (spike_pstrsv_ops.c:1186)."""
        pad = 16
        bb = np.zeros(self.m + 2 * pad)
        xx = np.zeros(self.m + 2 * pad)
        bb[pad:pad + self.m] = b
        f = self.lib()._spike_pstrsv_solve if timed else self.lib().spike_pstrsv_solve
        f(b"U", self.m, bb.ctypes.data + 8 * pad, xx.ctypes.data + 8 * pad, self.P)
        return xx[pad:pad + self.m].copy()

    def set_partitions(self, starts, ends) -> None:
        """Caller-set partition bounds for the next preproc (IS_MATRIX_PARTITIONED,
        src/matrix_partitioning.c:23-35; the solve reads partition_numRows too)."""
        I = ctypes.c_int32
        for name, vals in (("partition_starts", starts), ("partition_ends", ends),
                           ("partition_numRows", np.asarray(ends) - np.asarray(starts))):
            base = ctypes.addressof(self._sym(name, I))
            for k, v in enumerate(vals):
                I.from_address(base + 4 * k).value = int(v)
        self.set_flag("IS_MATRIX_PARTITIONED", 1)

    def reorder(self, A, P: int, uplo: str, part) -> tuple:
        """The reference's matrixReordering (src/matrix_reordering.c:83-305) on the
        full matrix A (symmetric pattern, symm 'Y'), with its METIS call answered
        by `part` (ref/reorder_stubs.c).  Returns (a, ia, ja, starts, ends,
        numRows) and leaves IS_MATRIX_PARTITIONED set for the next preproc."""
        lib = self.lib()
        lib.mkl_malloc.restype = ctypes.c_void_p
        lib.mkl_malloc.argtypes = [ctypes.c_size_t, ctypes.c_int]
        lib.spk_ref_set_partition.argtypes = [ctypes.c_void_p, ctypes.c_int]
        lib.matrixReordering.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_char, ctypes.c_char, ctypes.c_char_p]
        n = int(A.m)
        pv = _i32(part)
        lib.spk_ref_set_partition(pv.ctypes.data, n)
        ptrs = []
        for arr, ct in ((_f64(A.a), ctypes.c_double), (_i32(A.ia), ctypes.c_int32), (_i32(A.ja), ctypes.c_int32)):
            p = lib.mkl_malloc(max(arr.nbytes, 8), 64)
            ctypes.memmove(p, arr.ctypes.data, arr.nbytes)
            ptrs.append(ctypes.c_void_p(p))
        lib.matrixReordering(ctypes.byref(ptrs[0]), ctypes.byref(ptrs[1]), ctypes.byref(ptrs[2]), n, int(P),
                             uplo.encode()[:1], b"Y", None)

        def read(p, ct, count):
            return np.ctypeslib.as_array((ct * count).from_address(p.value)).copy()

        ia = read(ptrs[1], ctypes.c_int32, n + 1)
        nnz = int(ia[n])
        out = (read(ptrs[0], ctypes.c_double, nnz), ia, read(ptrs[2], ctypes.c_int32, nnz))
        I = ctypes.c_int32
        bounds = tuple(self._arr(k, I, P) for k in ("partition_starts", "partition_ends", "partition_numRows"))
        return out + bounds

    def solve_raw(self, bbuf_addr: int, xbuf_addr: int, timed: bool = True) -> None:
        f = self.lib()._spike_pstrsv_solve if timed else self.lib().spike_pstrsv_solve
        f(b"U", self.m, bbuf_addr, xbuf_addr, self.P)

    def _arr(self, name, ctype, count):
        if count <= 0:
            return np.zeros(0, dtype=np.dtype(ctype))
        addr = ctypes.addressof(self._sym(name, ctype))
        return np.ctypeslib.as_array((ctype * count).from_address(addr)).copy()

    def _ptr_arr(self, name, ctype, count):
        if count <= 0:
            return np.zeros(0, dtype=np.dtype(ctype))
        addr = ctypes.c_void_p.in_dll(self.lib(), name).value
        return np.ctypeslib.as_array((ctype * count).from_address(addr)).copy()

    def structure(self) -> dict:
        n, P = self.m, self.P
        I, C, Q, Dd = ctypes.c_int32, ctypes.c_int8, ctypes.c_int64, ctypes.c_double
        out = {}
        for k in ["partition_starts", "partition_ends", "partition_numRows", "starts_D", "ends_D",
                  "starts_R", "ends_R", "numRows_S", "numCols_S", "start_intervals",
                  "end_intervals", "starts_D0", "ends_D0", "starts_D1", "ends_D1", "starts_D2",
                  "ends_D2", "starts_mapR", "ends_mapR"]:
            out[k] = self._arr(k, I, P)
        for k in ["hasDependences", "hasReflections", "hasToCalculateSs", "isOptimizeds"]:
            out[k] = self._arr(k, C, P)
        out["starts_S"] = self._arr("starts_S", Q, P)
        out["ends_S"] = self._arr("ends_S", Q, P)
        out["ID"] = self._arr("ID", I, 2 * n + 1)
        nd = int(out["ID"][2 * n])
        out["D"] = self._arr("D", Dd, nd)
        out["JD"] = self._arr("JD", I, nd)
        split = (out["hasReflections"] != 0) | (out["isOptimizeds"] != 0)
        rows = max([0] + [int(v) for v in out["ends_D0"][out["hasReflections"] != 0]]
                   + [int(v) for v in out["ends_D1"][split]] + [int(v) for v in out["ends_D2"][split]])
        out["IT2"] = self._arr("IT2", I, rows + 1)
        n2 = int(out["IT2"][rows])
        out["T2"] = self._arr("T2", Dd, n2)
        out["JT2"] = self._arr("JT2", I, n2)
        out["mapR"] = self._ptr_arr("mapR", I, int(out["numCols_S"].sum()))
        out["S"] = self._ptr_arr("S", Dd, int(out["ends_S"][P - 1])) if self._sym("isReducedSystemNecessary", C).value else np.zeros(0)
        nred = self._sym("numRowsReducedSystem", I).value
        rss = self._sym("reducedSystemSolverStart", I).value
        out["mapReducedX"] = self._arr("mapReducedX", I, nred)
        out["IT"] = self._arr("IT", I, rss + 1)
        nt = int(out["IT"][rss]) if rss >= 0 else 0
        out["T"] = self._arr("T", Dd, nt)
        out["JT"] = self._arr("JT", I, nt)
        out["numRowsReducedSystem"] = nred
        out["numNnzsReducedSystem"] = self._sym("numNnzsReducedSystem", I).value
        out["reducedSystemSolverStart"] = rss
        out["isReducedSystemNecessary"] = self._sym("isReducedSystemNecessary", C).value
        return out
