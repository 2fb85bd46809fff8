"""Triangular factor pairs: x = (L L^T)^{-1} b as a forward solve with L
(uplo 'L') and a backward solve with L^T (uplo 'U'), the application of an
incomplete-Cholesky preconditioner.  Each triangle is one resident preprocessed
system; the FP32 form solves each triangle with FP32 values and FP64
refinement to scaled residual <= 1e-12 (spk_solve_batch mode 1).

Benchmark workload: the IC(0)-style factor of the 7-point 3-D Laplacian on an
n^3 grid (<= 4 nonzeros per row of L; L_ii = sqrt(6), off-diagonals
-1/sqrt(6) x U(0.9, 1.1), seeded), one and 32 right-hand sides, FP64 and FP32 +
refinement, against the plain FP64 solve pair.  The factor couples rows n^2
apart, so the dense spikes hold about m * n^2 values whatever the partition
count; the spike storage bound (16 GiB for three copies, as the reference's
MEMSIZE) admits n <= 48 (m = 110,592, 255M spike values).  At n = 128
(m = 2,097,152) the spikes would hold 34G values (275 GB), beyond the bound and
beyond one GPU's memory.

    python -m spike_pstrsv_b200.pair [--n 48 --nparts 8]
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import synth
from .capi import System

MODE_FP64 = 0
MODE_FP32_IR = 1


class TriangularPair:
    def __init__(self, L, nparts: int, U=None):
        U = synth.transpose(L) if U is None else U
        self.m = L.m
        self.lower = System().preproc(L.a, L.ia, L.ja, L.m, nparts, "L", 1)
        self.upper = System().preproc(U.a, U.ia, U.ja, U.m, nparts, "U", 1)

    def solve(self, B, X, mode: int = MODE_FP32_IR, tol: float = 1e-12, maxit: int = 8, stream: int = 0,
              Y=None, want_resid: bool = True):
        """B, X (and the intermediate Y): CUDA tensors (nrhs, m).  Returns the
        refinement steps and scaled residuals of the two triangular solves."""
        import torch
        Y = torch.empty_like(B) if Y is None else Y
        i1, r1 = self.lower.solve_batch(B, Y, mode=mode, tol=tol, maxit=maxit, stream=stream, want_resid=want_resid)
        i2, r2 = self.upper.solve_batch(Y, X, mode=mode, tol=tol, maxit=maxit, stream=stream, want_resid=want_resid)
        return (i1, i2), (r1, r2)


def run(n: int = 48, nparts: int = 8, reps: int = 10):
    import torch
    L = synth.ic0_laplace3d_lower(n)
    U = synth.transpose(L)
    m = L.m
    out = {"workload": f"IC(0)-style L and L^T of the 7-point Laplacian on {n}^3 (m={m}, nnz(L)={L.nnz}), "
                       f"nparts={nparts}", "m": m, "nnz_L": int(L.nnz), "runs": []}
    pair = TriangularPair(L, nparts, U)
    st = torch.cuda.current_stream()
    for k in (1, 32):
        rng = np.random.default_rng(k)
        Xt = rng.uniform(-1, 1, size=(k, m))
        B = np.stack([synth.spmv(L, synth.spmv(U, Xt[i])) for i in range(k)])
        dB = torch.from_numpy(B).cuda()
        dX, dY = torch.zeros_like(dB), torch.zeros_like(dB)
        for mode in (MODE_FP64, MODE_FP32_IR):
            steps, res = pair.solve(dB, dX, mode=mode, Y=dY, stream=st.cuda_stream)
            fixed = max(steps)
            for _ in range(2):
                pair.solve(dB, dX, mode=mode, tol=-1.0, maxit=fixed, Y=dY, stream=st.cuda_stream, want_resid=False)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for _ in range(reps):
                pair.solve(dB, dX, mode=mode, tol=-1.0, maxit=fixed, Y=dY, stream=st.cuda_stream, want_resid=False)
            e1.record(st)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / reps
            steps, res = pair.solve(dB, dX, mode=mode, tol=-1.0, maxit=fixed, Y=dY, stream=st.cuda_stream)
            X = dX.cpu().numpy()
            err = max(float(np.linalg.norm(X[i] - Xt[i]) / np.linalg.norm(Xt[i])) for i in range(k))
            out["runs"].append({"rhs": k, "mode": "fp64" if mode == MODE_FP64 else "fp32_ir",
                                "refinement_steps": list(steps), "ms_per_pair_solve": ms,
                                "pair_solves_per_s": k * 1e3 / ms, "scaled_residuals": list(res),
                                "rel_err_vs_x_true": err})
    base = {r["rhs"]: r["pair_solves_per_s"] for r in out["runs"] if r["mode"] == "fp64" and r["rhs"] == 1}
    for r in out["runs"]:
        r["vs_plain_fp64"] = r["pair_solves_per_s"] / base[1]
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=48)
    ap.add_argument("--nparts", type=int, default=8)
    args = ap.parse_args()
    print(json.dumps(run(args.n, args.nparts)))


if __name__ == "__main__":
    main()
