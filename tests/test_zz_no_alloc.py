"""spk_solve_batch_noalloc (fixed static scratch, no device allocation) against
spk_solve_batch in FP64, called through the C ABI twice in a row.

Named to be collected last; it also passes alone in a fresh process."""
import ctypes

import numpy as np
import pytest

import spike_pstrsv_b200 as spk
from spike_pstrsv_b200 import capi, synth

pytestmark = pytest.mark.gpu

SCRATCH = 1 << 19  # FP64 values in the library's static scratch
SPK_ERR_TOO_LARGE = -6


def _noalloc():
    f = capi.lib().spk_solve_batch_noalloc
    vp = ctypes.c_void_p
    f.argtypes = [vp, ctypes.c_int, vp, ctypes.c_longlong, vp, ctypes.c_longlong, vp]
    f.restype = ctypes.c_int
    return f


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda:0")


def _call(S, dB, dX):
    import torch
    rc = _noalloc()(S.h, dB.shape[0], ctypes.c_void_p(dB.data_ptr()), dB.stride(0),
                    ctypes.c_void_p(dX.data_ptr()), dX.stride(0), None)
    torch.cuda.synchronize()
    return rc


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("case", ["poisson_L_40", "banded_U_13"])
def test_noalloc_matches_batch_solve_twice(case):
    import torch
    if case == "poisson_L_40":
        A, uplo, nparts, nrhs = synth.poisson2d_lower(128), "L", 4, 40     # groups 32 + 8
    else:
        A, uplo, nparts, nrhs = synth.transpose(synth.banded_lower(60000, seed=21)), "U", 16, 13  # 8 + 4 + 1
    Xt, B = synth.make_rhs(A, seed=9, nrhs=nrhs)
    S = spk.System().preproc(A.a, A.ia, A.ja, A.m, nparts, uplo, 1)
    assert S.scalar("ell") == 1
    dB = _dev(B)
    dref = torch.zeros_like(dB)
    S.solve_batch(dB, dref, mode=0, want_resid=False)
    ref = dref.cpu().numpy()
    for call in range(2):
        dX = torch.zeros_like(dB)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        rc = _call(S, dB, dX)
        assert rc == 0, capi.lib().spk_last_error().decode()
        if call == 1:
            assert torch.cuda.mem_get_info()[0] == free0
        X = dX.cpu().numpy()
        for k in range(nrhs):
            assert _rel(X[k], ref[k]) <= 1e-13
            assert _rel(X[k], Xt[k]) <= 1e-11
    assert np.array_equal(dB.cpu().numpy(), B)


def test_noalloc_rejects_systems_beyond_the_scratch():
    import torch
    A = synth.banded_lower(SCRATCH + 1000, seed=2)
    S = spk.System().preproc(A.a, A.ia, A.ja, A.m, 64, "L", 1)
    dB = torch.zeros((1, A.m), dtype=torch.float64, device="cuda:0")
    dX = torch.zeros_like(dB)
    assert _call(S, dB, dX) == SPK_ERR_TOO_LARGE
    assert "static scratch" in capi.lib().spk_last_error().decode()
