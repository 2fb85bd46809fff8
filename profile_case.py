"""A small, self-contained solve workload for profiler captures (ncu) of the
solve kernels.  Not part of the library: it drives the library the way a user
would, so that a capture sees only the solve's own launches.

    python profile_case.py --m 2097152 --P 512 --nrhs 1
        plain FP64 solves (spk_solve_device: k_chain_solve, or k_tile_solve with
        --no-chain)
    python profile_case.py --m 2097152 --P 512 --nrhs 32 --mode 1
        batched solves (spk_solve_batch; FP32 + one refinement step with mode 1)

The system is the banded lower-triangular workload (16 of the 64 preceding
columns per row) with m rows, solved with uplo 'L' and P partitions; --solves
calls follow one warm-up call.
"""
from __future__ import annotations

import argparse
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def main():
    import torch

    import spike_pstrsv_b200 as spk
    from spike_pstrsv_b200 import synth

    ap = argparse.ArgumentParser()
    ap.add_argument("--m", type=int, default=2097152)
    ap.add_argument("--P", type=int, default=512)
    ap.add_argument("--nrhs", type=int, default=1)
    ap.add_argument("--mode", type=int, default=0)
    ap.add_argument("--solves", type=int, default=3)
    ap.add_argument("--no-chain", action="store_true", help="the partition-based solve (SPK_DISABLE_CHAIN=1)")
    args = ap.parse_args()
    if args.no_chain:
        os.environ["SPK_DISABLE_CHAIN"] = "1"
    L = synth.banded_lower(args.m)
    S = spk.System().preproc(L.a, L.ia, L.ja, L.m, args.P, "L", 1)
    st = torch.cuda.current_stream()
    if args.nrhs == 1 and args.mode == 0:
        _, b = synth.make_rhs(L, seed=1)
        db = torch.from_numpy(b).cuda()
        dx = torch.zeros_like(db)
        for _ in range(1 + args.solves):
            S.solve_device(db.data_ptr(), dx.data_ptr(), st.cuda_stream)
    else:
        _, B = synth.make_rhs(L, seed=1, nrhs=args.nrhs)
        dB = torch.from_numpy(B).cuda()
        dX = torch.zeros_like(dB)
        for _ in range(1 + args.solves):
            S.solve_batch(dB, dX, mode=args.mode, tol=-1.0, maxit=1, stream=st.cuda_stream, want_resid=False)
    torch.cuda.synchronize()
    S.check()
    print("ok", args.m, args.P, args.nrhs, args.mode)


if __name__ == "__main__":
    main()
