"""ctypes binding of libspike_pstrsv_b200.so (include/spike_pstrsv.h).

The functions mirror the reference's C API one to one (src/spike_pstrsv.h:7-38):
same names, same argument order and meaning (``nthreads`` is the partition
count), same global flags.  Arrays may be numpy arrays (host memory) or CUDA
tensors/objects exposing ``data_ptr()`` (device memory); the library tells them
apart with cudaPointerGetAttributes.

There is no CPU fallback: importing the package works without a GPU, but every
call that computes needs the compiled library and a CUDA device, and raises
otherwise.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import build as _build

LIB_PATH = _build.LIB

_lib = None


class SpkError(RuntimeError):
    """A library call failed; ``code`` is the spk status code."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def lib() -> ctypes.CDLL:
    """Load the compiled library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run spike_pstrsv_b200.build.build() "
                               "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        vp, i, c, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_char, ctypes.c_double
        L.spike_pstrsv_preproc.argtypes = [vp, vp, vp, i, i, c]
        L._spike_pstrsv_preproc.argtypes = [vp, vp, vp, i, i, c]
        L.spike_pstrsv.argtypes = [c, i, vp, vp, vp, vp, vp, i]
        L.spike_pstrsv_solve.argtypes = [c, i, vp, vp, i]
        L._spike_pstrsv_solve.argtypes = [c, i, vp, vp, i]
        L.logPSTRSV3.argtypes = [i]
        L.spk_last_error.restype = ctypes.c_char_p
        L.spk_create.argtypes = [ctypes.POINTER(vp)]
        L.spk_destroy.argtypes = [vp]
        L.spk_preproc.argtypes = [vp, vp, vp, vp, i, i, c, i, vp, vp]
        L.spk_solve_device.argtypes = [vp, vp, vp, vp]
        L.spk_solve.argtypes = [vp, vp, vp]
        L.spk_debug_array.argtypes = [vp, ctypes.c_char_p, vp, ctypes.c_longlong,
                                      ctypes.POINTER(ctypes.c_longlong), ctypes.c_char_p]
        L.spk_debug_scalar.restype = ctypes.c_longlong
        L.spk_debug_scalar.argtypes = [vp, ctypes.c_char_p]
        L.spk_debug_set.argtypes = [vp, ctypes.c_char_p, ctypes.c_longlong]
        L.spk_chain_phase.argtypes = [vp, i, i, i, vp, vp, vp]
        L.spk_compact.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
        L.spk_legacy_system.restype = vp
        L.spk_set_truncation.argtypes = [vp, d]
        L.spk_check.argtypes = [vp]
        L.spk_set_profiling.argtypes = [vp, i]
        L.spk_solve_batch.argtypes = [vp, i, vp, ctypes.c_longlong, vp, ctypes.c_longlong, i, d, i, vp,
                                      ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)]
        L.spk_set_workspace.argtypes = [vp, vp, ctypes.c_longlong]
        L.spk_workspace_bytes.argtypes = [vp, i, i]
        L.spk_workspace_bytes.restype = ctypes.c_longlong
        L.spk_phase_times.argtypes = [vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_longlong)]
        _lib = L
    return _lib


def last_error() -> tuple[int, str]:
    L = lib()
    return int(L.spk_last_error_code()), (L.spk_last_error() or b"").decode()


def _check(rc: int) -> None:
    if rc != 0:
        code, msg = last_error()
        raise SpkError(rc, msg)


def _arr(x, dtype, keep: list, writable: bool = False):
    """Pointer to x: a device pointer for CUDA tensors, else a contiguous host copy/view."""
    if hasattr(x, "data_ptr") and getattr(x, "is_cuda", False):
        if not x.is_contiguous():
            raise ValueError("device arrays must be contiguous")
        return x.data_ptr()
    if hasattr(x, "data_ptr"):  # CPU tensor
        x = x.numpy()
    a = np.asarray(x)
    if a.dtype != dtype or not a.flags["C_CONTIGUOUS"]:
        if writable:
            raise ValueError(f"output array must be contiguous {np.dtype(dtype)}")
        a = np.ascontiguousarray(a, dtype=dtype)
    keep.append(a)
    return a.ctypes.data


def _uplo(u) -> bytes:
    return (u.encode() if isinstance(u, str) else bytes(u))[:1]


# ---- reference API -------------------------------------------------------------

def spike_pstrsv_preproc(a, ia, ja, n: int, nthreads: int, uplo: str = "U") -> None:
    keep: list = []
    lib().spike_pstrsv_preproc(_arr(a, np.float64, keep), _arr(ia, np.int32, keep),
                               _arr(ja, np.int32, keep), int(n), int(nthreads), _uplo(uplo))


def _spike_pstrsv_preproc(a, ia, ja, n: int, nthreads: int, uplo: str = "U") -> None:
    keep: list = []
    lib()._spike_pstrsv_preproc(_arr(a, np.float64, keep), _arr(ia, np.int32, keep),
                                _arr(ja, np.int32, keep), int(n), int(nthreads), _uplo(uplo))


def spike_pstrsv(uplo: str, m: int, a, ia, ja, b, x, nthreads: int) -> None:
    keep: list = []
    lib().spike_pstrsv(_uplo(uplo), int(m), _arr(a, np.float64, keep), _arr(ia, np.int32, keep),
                       _arr(ja, np.int32, keep), _arr(b, np.float64, keep, True),
                       _arr(x, np.float64, keep, True), int(nthreads))


def spike_pstrsv_solve(uplo: str, m: int, b, x, nthreads: int) -> None:
    keep: list = []
    lib().spike_pstrsv_solve(_uplo(uplo), int(m), _arr(b, np.float64, keep, True),
                             _arr(x, np.float64, keep, True), int(nthreads))


def _spike_pstrsv_solve(uplo: str, m: int, b, x, nthreads: int) -> None:
    keep: list = []
    lib()._spike_pstrsv_solve(_uplo(uplo), int(m), _arr(b, np.float64, keep, True),
                              _arr(x, np.float64, keep, True), int(nthreads))


def free_PSTRSV3() -> None:
    lib().free_PSTRSV3()


def logPSTRSV3(nthreads: int) -> None:
    lib().logPSTRSV3(int(nthreads))


_FLAGS = ("PSTRSV_VERBOSE", "FORCE_LOAD_BALANCE", "IS_MATRIX_PARTITIONED", "SPK_CLOBBER_B", "SPK_EXACT")
TIMERS = ("memoryAlloc_timer_pstrsv3", "preprocessD_timer_pstrsv3", "preprocessR_timer_pstrsv3",
          "setDependents_timer_pstrsv3", "preprocessS_timer_pstrsv3",
          "preprocessMappings_timer_pstrsv3", "produceCompressedR_timer_pstrsv3",
          "produceS_timer_pstrsv3", "produceReducedSystem_timer_pstrsv3", "init_vars_pstrsv3",
          "reduced_solver_timer_pstrsv3")


def set_flag(name: str, value: int) -> None:
    if name not in _FLAGS:
        raise KeyError(name)
    ctypes.c_int8.in_dll(lib(), name).value = int(value)


def get_flag(name: str) -> int:
    return int(ctypes.c_int8.in_dll(lib(), name).value)


def get_global(name: str, index: int | None = None):
    """Read an exported scalar/array global (timers, partition bounds, numRowsReducedSystem)."""
    if name in ("partition_starts", "partition_ends", "partition_numRows"):
        base = ctypes.addressof(ctypes.c_int32.in_dll(lib(), name))
        return ctypes.c_int32.from_address(base + 4 * (index or 0)).value
    if name == "numRowsReducedSystem":
        return ctypes.c_int32.in_dll(lib(), name).value
    if index is not None:
        base = ctypes.addressof(ctypes.c_double.in_dll(lib(), name))
        return ctypes.c_double.from_address(base + 8 * index).value
    return ctypes.c_double.in_dll(lib(), name).value


def set_partitions(starts, ends) -> None:
    """Fill partition_starts/ends and raise IS_MATRIX_PARTITIONED (the reordering path)."""
    L = lib()
    for name, vals in (("partition_starts", starts), ("partition_ends", ends)):
        base = ctypes.addressof(ctypes.c_int32.in_dll(L, name))
        for k, v in enumerate(vals):
            ctypes.c_int32.from_address(base + 4 * k).value = int(v)
    set_flag("IS_MATRIX_PARTITIONED", 1)


# ---- handle API ------------------------------------------------------------------

_DT = {"d": np.float64, "i": np.int32, "q": np.int64, "c": np.int8}


def _debug_array(h, name: str) -> np.ndarray:
    L = lib()
    cnt = ctypes.c_longlong()
    ty = ctypes.create_string_buffer(2)
    _check(L.spk_debug_array(h, name.encode(), None, 0, ctypes.byref(cnt), ty))
    out = np.zeros(cnt.value, dtype=_DT[ty.value.decode()])
    if cnt.value:
        _check(L.spk_debug_array(h, name.encode(), out.ctypes.data, cnt.value, ctypes.byref(cnt), ty))
    return out


class System:
    """One preprocessed matrix (spk_system)."""

    def __init__(self):
        h = ctypes.c_void_p()
        _check(lib().spk_create(ctypes.byref(h)))
        self.h = h
        self.n = 0
        self.uplo = "U"

    def close(self):
        if self.h:
            lib().spk_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def preproc(self, a, ia, ja, n: int, nparts: int, uplo: str = "U", flb: int = 1,
                starts=None, ends=None) -> "System":
        keep: list = []
        st = _arr(starts, np.int32, keep) if starts is not None else None
        en = _arr(ends, np.int32, keep) if ends is not None else None
        _check(lib().spk_preproc(self.h, _arr(a, np.float64, keep), _arr(ia, np.int32, keep),
                                 _arr(ja, np.int32, keep), int(n), int(nparts), _uplo(uplo),
                                 int(flb), st, en))
        self.n = int(n)
        self.uplo = uplo.upper() if isinstance(uplo, str) else chr(uplo[0]).upper()
        return self

    def set_truncation(self, tau: float) -> "System":
        """Spike truncation threshold (default 2^-60); tau < 0 = exact mode."""
        _check(lib().spk_set_truncation(self.h, float(tau)))
        return self

    def solve_batch(self, B, X, mode: int = 0, tol: float = 1e-12, maxit: int = 5, stream: int = 0,
                    want_resid: bool = True):
        """Batched solve of the columns of B (CUDA tensors, shape (nrhs, n): row k is
        right-hand side k).  mode 0: FP64; mode 1: FP32 solves + FP64 refinement.
        Returns (corrections applied, largest scaled residual or None)."""
        nrhs, n = B.shape
        it = ctypes.c_int(0)
        r = ctypes.c_double(-1.0)
        _check(lib().spk_solve_batch(self.h, int(nrhs), ctypes.c_void_p(B.data_ptr()), int(B.stride(0)),
                                     ctypes.c_void_p(X.data_ptr()), int(X.stride(0)), int(mode), float(tol),
                                     int(maxit), ctypes.c_void_p(stream), ctypes.byref(it),
                                     ctypes.byref(r) if want_resid else None))
        return it.value, (r.value if want_resid else None)

    def set_workspace(self, ws=None) -> "System":
        """Lend device memory (a CUDA tensor, 256-byte aligned) for the batched
        solves' work columns; None detaches it."""
        if ws is None:
            _check(lib().spk_set_workspace(self.h, None, 0))
        else:
            _check(lib().spk_set_workspace(self.h, ctypes.c_void_p(ws.data_ptr()),
                                           int(ws.numel() * ws.element_size())))
        self._ws = ws
        return self

    def workspace_bytes(self, mode: int = 1, with_residual: bool = True) -> int:
        return int(lib().spk_workspace_bytes(self.h, int(mode), int(with_residual)))

    def set_profiling(self, on: bool = True) -> "System":
        _check(lib().spk_set_profiling(self.h, int(on)))
        return self

    def phase_times(self):
        """(ms of phase 1, phase 2, phase 3+4 accumulated, number of solves); resets."""
        ms = (ctypes.c_double * 3)()
        n = ctypes.c_longlong()
        _check(lib().spk_phase_times(self.h, ms, ctypes.byref(n)))
        return [ms[0], ms[1], ms[2]], n.value

    def check(self) -> None:
        """Wait for the system's stream and raise on a device-side failure."""
        _check(lib().spk_check(self.h))

    def solve(self, b, x=None):
        """Synchronous solve; host (numpy) or device (CUDA tensor) arrays."""
        keep: list = []
        if x is None:
            x = np.zeros(self.n)
        _check(lib().spk_solve(self.h, _arr(b, np.float64, keep), _arr(x, np.float64, keep, True)))
        return x

    def solve_device(self, b_ptr: int, x_ptr: int, stream: int = 0) -> None:
        """Asynchronous solve on device pointers and a cudaStream_t handle."""
        _check(lib().spk_solve_device(self.h, ctypes.c_void_p(b_ptr), ctypes.c_void_p(x_ptr),
                                      ctypes.c_void_p(stream)))

    def array(self, name: str) -> np.ndarray:
        return _debug_array(self.h, name)

    def scalar(self, name: str) -> int:
        return int(lib().spk_debug_scalar(self.h, name.encode()))

    def chain_phase(self, phase: int, row_lo: int, row_hi: int, b_ptr: int, x_ptr: int, stream: int = 0) -> None:
        """One phase (1 or 4) of the chain solve over U rows [row_lo, row_hi), on
        device pointers (spk_chain_phase)."""
        _check(lib().spk_chain_phase(self.h, int(phase), int(row_lo), int(row_hi), ctypes.c_void_p(b_ptr),
                                     ctypes.c_void_p(x_ptr), ctypes.c_void_p(stream)))

    def compact(self) -> int:
        """Release the device pools the chain solves never read (spk_compact);
        returns the bytes released."""
        freed = ctypes.c_longlong(0)
        _check(lib().spk_compact(self.h, ctypes.byref(freed)))
        return int(freed.value)

    def tune(self, name: str, value: int) -> "System":
        """Chain-solver knobs (spk_tune): "rows" and "batch_rows" (rows per chain
        task of the one-right-hand-side and batched solves), "stages" (2 or 3 tiles
        staged ahead), "batch_path" (1 chain, 0 partition kernels, -1 automatic)."""
        L = lib()
        L.spk_tune.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_longlong]
        _check(L.spk_tune(self.h, name.encode(), int(value)))
        return self

    def debug_set(self, name: str, value: int) -> "System":
        """Test hooks (spk_debug_set): "fail_waits" makes the solve kernels report a
        failed bounded wait until the failure has been reported once."""
        _check(lib().spk_debug_set(self.h, name.encode(), int(value)))
        return self

    def structure(self) -> dict:
        from_names = [
            "partition_starts", "partition_ends", "partition_numRows",
            "D", "ID", "JD", "starts_D", "ends_D", "starts_R", "ends_R",
            "hasDependences", "hasReflections", "hasToCalculateSs", "isOptimizeds",
            "numRows_S", "numCols_S", "starts_S", "ends_S", "start_intervals", "end_intervals",
            "T2", "IT2", "JT2", "starts_D0", "ends_D0", "starts_D1", "ends_D1", "starts_D2",
            "ends_D2", "mapR", "starts_mapR", "ends_mapR", "S", "mapReducedX", "T", "IT", "JT"]
        out = {k: self.array(k) for k in from_names}
        for k in ("numRowsReducedSystem", "numNnzsReducedSystem", "reducedSystemSolverStart",
                  "isReducedSystemNecessary"):
            out[k] = self.scalar(k)
        return out


def legacy_structure() -> dict:
    """Structure of the system held by the reference-API entry points."""
    h = lib().spk_legacy_system()
    if not h:
        raise SpkError(-5, "no preprocessed system")
    s = System.__new__(System)
    s.h = ctypes.c_void_p(h)
    s.n = 0
    out = s.structure()
    s.h = None  # not owned
    return out


# ---- partition-aware reordering (src/matrix_reordering.c) --------------------------

def _libc() -> ctypes.CDLL:
    c = ctypes.CDLL(None)
    c.malloc.restype = ctypes.c_void_p
    c.malloc.argtypes = [ctypes.c_size_t]
    c.free.argtypes = [ctypes.c_void_p]
    return c


def reorder_plan(ia, ja, n: int, nparts: int):
    """The reordering's partitioner (host code): (order, part), order[q] = the row
    at position q of the reverse Cuthill-McKee order, part[r] = partition of row r."""
    L = lib()
    ia = np.ascontiguousarray(ia, dtype=np.int32)
    ja = np.ascontiguousarray(ja, dtype=np.int32)
    order = np.zeros(n, dtype=np.int32)
    part = np.zeros(n, dtype=np.int32)
    vp = ctypes.c_void_p
    L.spk_reorder_plan.argtypes = [ctypes.c_int, vp, vp, ctypes.c_int, vp, vp]
    _check(L.spk_reorder_plan(int(n), ia.ctypes.data, ja.ctypes.data, int(nparts), order.ctypes.data,
                              part.ctypes.data))
    return order, part


def reorder(a, ia, ja, n: int, nparts: int, uplo: str = "U", legacy: bool = False):
    """Reorder the full host CSR (a, ia, ja) for nparts partitions and keep one
    triangle.  legacy=False: spk_reorder, returns (a, ia, ja, perm).  legacy=True:
    the reference entry point matrixReordering (symm 'Y', no file), returns
    (a, ia, ja, None) with the partition globals set and IS_MATRIX_PARTITIONED
    raised for the next spike_pstrsv_preproc."""
    L, C = lib(), _libc()
    arrs = (np.ascontiguousarray(a, dtype=np.float64), np.ascontiguousarray(ia, dtype=np.int32),
            np.ascontiguousarray(ja, dtype=np.int32))
    ptrs = []
    for x in arrs:  # the library frees the inputs with free() and returns malloc'd arrays
        p = C.malloc(max(x.nbytes, 8))
        if not p:
            raise MemoryError("malloc failed")
        ctypes.memmove(p, x.ctypes.data, x.nbytes)
        ptrs.append(ctypes.c_void_p(p))
    refs = [ctypes.byref(p) for p in ptrs]
    perm = None
    if legacy:
        L.matrixReordering.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int, ctypes.c_int, ctypes.c_char,
                                                               ctypes.c_char, ctypes.c_char_p]
        L.matrixReordering(*refs, int(n), int(nparts), _uplo(uplo), b"Y", None)
    else:
        perm = np.zeros(n, dtype=np.int32)
        L.spk_reorder.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int, ctypes.c_int, ctypes.c_char,
                                                          ctypes.c_void_p]
        rc = L.spk_reorder(*refs, int(n), int(nparts), _uplo(uplo), perm.ctypes.data)
        if rc != 0:
            for p in ptrs:
                C.free(p)
            _check(rc)

    def take(p, ct, count):
        out = np.ctypeslib.as_array((ct * max(count, 1)).from_address(p.value))[:count].copy()
        C.free(p)
        return out

    ia_o = take(ptrs[1], ctypes.c_int32, n + 1)
    nnz = int(ia_o[n])
    return take(ptrs[0], ctypes.c_double, nnz), ia_o, take(ptrs[2], ctypes.c_int32, nnz), perm
