"""ctypes binding of the serving loop (spk_server_* in include/spike_pstrsv.h).

The server keeps preprocessed systems resident in HBM under a byte budget (LRU
eviction of idle systems), batches queued solve requests of the same matrix (up
to 32 right-hand sides per batch) and runs batches of different matrices
concurrently on its worker streams.  Requests carry host arrays; the binding
keeps them alive until the request completes.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from .capi import SpkError, lib

MODE_FP64 = 0
MODE_FP32_IR = 1
STATS = ("resident_bytes", "staging_bytes", "resident_systems", "evictions", "preprocessings", "batches",
         "rhs_batched", "completed", "budget", "nomem_retries", "rechecks", "us_stage_in", "us_solve",
         "us_stage_out", "us_preprocess", "compactions")

_bound = False


def _bind():
    global _bound
    if _bound:
        return lib()
    L = lib()
    vp, i, ll, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_double
    L.spk_server_create.argtypes = [ctypes.POINTER(vp), ll, i]
    L.spk_server_destroy.argtypes = [vp]
    L.spk_server_put_matrix.argtypes = [vp, i, vp, vp, vp, i, i, ctypes.c_char]
    L.spk_server_submit.argtypes = [vp, i, i, vp, vp, i, ctypes.POINTER(ll)]
    L.spk_server_wait.argtypes = [vp, ll, ctypes.POINTER(d), ctypes.POINTER(d), ctypes.POINTER(i),
                                  ctypes.POINTER(i)]
    L.spk_server_stats.argtypes = [vp, ctypes.POINTER(ll), i]
    _bound = True
    return L


def _check(rc: int):
    if rc != 0:
        raise SpkError(rc, lib().spk_last_error().decode())


@dataclass
class Result:
    x: np.ndarray          # (nrhs, n) solutions
    latency_s: float       # submit to result in host memory
    scaled_residual: float  # of the request's batch
    refinement_steps: int
    batch_rhs: int         # right-hand sides in the batch that served it


class Ticket:
    def __init__(self, server: "Server", ticket: int, b: np.ndarray, x: np.ndarray):
        self.server, self.ticket, self._b, self.x = server, ticket, b, x

    def wait(self) -> Result:
        lat, res = ctypes.c_double(), ctypes.c_double()
        it, kb = ctypes.c_int(), ctypes.c_int()
        _check(_bind().spk_server_wait(self.server.h, self.ticket, ctypes.byref(lat), ctypes.byref(res),
                                       ctypes.byref(it), ctypes.byref(kb)))
        return Result(self.x, lat.value, res.value, it.value, kb.value)


class Server:
    """Serving loop on the current CUDA device."""

    def __init__(self, hbm_budget_bytes: int, slots: int = 4):
        L = _bind()
        h = ctypes.c_void_p()
        _check(L.spk_server_create(ctypes.byref(h), int(hbm_budget_bytes), int(slots)))
        self.h = h
        self.n = {}

    def close(self):
        if self.h:
            _bind().spk_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def put_matrix(self, mid: int, a, ia, ja, n: int, nparts: int, uplo: str = "L"):
        a = np.ascontiguousarray(a, np.float64)
        ia = np.ascontiguousarray(ia, np.int32)
        ja = np.ascontiguousarray(ja, np.int32)
        _check(_bind().spk_server_put_matrix(self.h, int(mid), a.ctypes.data, ia.ctypes.data, ja.ctypes.data,
                                             int(n), int(nparts), uplo.encode()))
        self.n[mid] = int(n)

    def submit(self, mid: int, B, mode: int = MODE_FP32_IR) -> Ticket:
        """B: (nrhs, n) or (n,) host array of right-hand sides."""
        b = np.ascontiguousarray(np.atleast_2d(B), np.float64)
        nrhs, n = b.shape
        if n != self.n.get(mid, -1):
            raise ValueError(f"right-hand sides of length {n} for matrix {mid} of size {self.n.get(mid)}")
        x = np.empty_like(b)
        t = ctypes.c_longlong()
        _check(_bind().spk_server_submit(self.h, int(mid), nrhs, b.ctypes.data, x.ctypes.data, int(mode),
                                         ctypes.byref(t)))
        return Ticket(self, t.value, b, x)

    def stats(self) -> dict:
        out = (ctypes.c_longlong * len(STATS))()
        _check(_bind().spk_server_stats(self.h, out, len(STATS)))
        return dict(zip(STATS, list(out)))
