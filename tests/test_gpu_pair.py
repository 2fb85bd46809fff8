"""Forward-then-backward solve with an IC(0)-style factor pair (L, L^T): FP64 and
FP32 + FP64 refinement against the sequential FP64 oracle."""
import numpy as np
import pytest

import oracle
from spike_pstrsv_b200 import pair, synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", [pair.MODE_FP64, pair.MODE_FP32_IR])
@pytest.mark.parametrize("nrhs", [1, 5])
def test_pair_matches_the_sequential_oracle(mode, nrhs):
    import torch
    L = synth.ic0_laplace3d_lower(24, seed=1)
    U = synth.transpose(L)
    P = pair.TriangularPair(L, 8, U)
    rng = np.random.default_rng(nrhs)
    Xt = rng.uniform(-1, 1, size=(nrhs, L.m))
    B = np.stack([synth.spmv(L, synth.spmv(U, Xt[i])) for i in range(nrhs)])
    dB = torch.from_numpy(B).cuda()
    dX = torch.zeros_like(dB)
    steps, res = P.solve(dB, dX, mode=mode)
    X = dX.cpu().numpy()
    for r in res:
        assert r <= 1e-12
    if mode == pair.MODE_FP32_IR:
        assert all(1 <= s <= 4 for s in steps)
    for i in range(nrhs):
        y = oracle.sequential_solve(L, B[i], "L")
        x = oracle.sequential_solve(U, y, "U")
        tol = 1e-13 if mode == pair.MODE_FP64 else 1e-12
        assert np.abs(X[i] - x).max() / np.abs(x).max() <= tol
        assert np.abs(X[i] - Xt[i]).max() <= 1e-10
