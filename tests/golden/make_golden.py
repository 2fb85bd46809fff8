"""Generate the golden fixtures in this folder from the reference itself.

Runs the reference's own sources (oracle/_ref/libspike_ref.so, built by
``make -C oracle ref`` from the reference tree) through its C API and records,
per case: the input CSR, the partition count, FORCE_LOAD_BALANCE, a right-hand
side, the reference's x, and its preprocessing state (every array of the
reference's globals that the structure tests compare).

* ``small_*.npz``  full arrays (small matrices).
* ``digest.json``  SHA-256 of every structure array plus the scalar fields, for
  the benchmark-sized cases (Poisson 128x128 at 4 partitions, banded 65,536 rows,
  and the full banded workload of 4,194,304 rows).

'L' cases run the reference's 'U' path on the reversal mirror J L J (the
reference's own 'L' path is unimplemented, src/spike_pstrsv.c:234-237).

* ``--full``       adds the full-size banded cases (m = 4,194,304; 'L' and 'U' at
  16, 64, 256 and 1024 partitions) to ``digest.json`` and stores the
  reference's x at sampled rows in ``full_x_samples.npz`` (a few minutes and
  ~25 GB of host memory: the reference keeps its pools in static arrays).

Usage: python tests/golden/make_golden.py [--full]   (needs the reference tree)
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import oracle  # noqa: E402
from cases import rand_upper  # noqa: E402
from spike_pstrsv_b200 import synth  # noqa: E402


def run_reference(A, P, uplo, flb, b):
    R = oracle.Reference()
    U = A if uplo == "U" else synth.mirror(A)
    R.preproc(U, P, flb=flb)
    st = R.structure()
    bu = b if uplo == "U" else b[::-1].copy()
    x = R.solve(bu)
    if uplo == "L":
        x = x[::-1].copy()
    return st, x


def digest(arr: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(arr).tobytes()).hexdigest()


def small_cases():
    out = []
    L = synth.poisson2d_lower(32)
    out.append(("small_poisson32_L_P4", L, 4, "L", 1))
    out.append(("small_poisson32_U_P5_flb0", synth.transpose(L), 5, "U", 0))
    B = synth.banded_lower(1024, seed=3)
    out.append(("small_banded1024_L_P8", B, 8, "L", 1))
    out.append(("small_banded1024_U_P3", synth.transpose(B), 3, "U", 1))
    for seed, m, P, band, dens, far, iso in [
        (0, 97, 13, 12, 0.4, 0.1, {2, 6, 10, 12}),   # isolated blocks kept split (INF sum wraps)
        (3, 132, 5, 20, 0.3, 0.0, {4}),               # isolated last block, decision reverted
        (17, 395, 23, 30, 0.5, 0.01, None),
        (21, 85, 9, 8, 0.6, 0.0, {0, 1, 6}),          # isolated first blocks
        (40, 60, 60, 3, 0.9, 0.1, None),              # one row per partition
    ]:
        A = rand_upper(m, dens, band, far, seed, iso, P)
        out.append((f"small_rand{seed}_U_P{P}", A, P, "U", 1))
    return out


def main():
    if not oracle.Reference.available():
        raise SystemExit("oracle/_ref/libspike_ref.so is missing: make -C oracle ref")
    for name, A, P, uplo, flb in small_cases():
        x_true, b = synth.make_rhs(A, seed=0)
        st, x = run_reference(A, P, uplo, flb, b)
        arrays = {f"s_{k}": v for k, v in st.items() if isinstance(v, np.ndarray)}
        scalars = {f"c_{k}": np.int64(v) for k, v in st.items() if not isinstance(v, np.ndarray)}
        np.savez_compressed(os.path.join(HERE, name + ".npz"), ia=A.ia, ja=A.ja, a=A.a, b=b, x_ref=x,
                            meta=np.array([A.m, P, flb, ord(uplo)], dtype=np.int64), **arrays, **scalars)
        print(name, "saved")
    dig = {}
    L = synth.poisson2d_lower(128)
    big = [("poisson128_L_P4", L, 4, "L", 1), ("poisson128_U_P4", synth.transpose(L), 4, "U", 1)]
    Bl = synth.banded_lower(65536, seed=0)
    big += [("banded65536_L_P16", Bl, 16, "L", 1), ("banded65536_L_P64_flb0", Bl, 64, "L", 0),
            ("banded65536_U_P256", synth.transpose(Bl), 256, "U", 1)]
    for name, A, P, uplo, flb in big:
        x_true, b = synth.make_rhs(A, seed=0)
        st, x = run_reference(A, P, uplo, flb, b)
        rec = {"m": int(A.m), "nnz": int(A.nnz), "P": P, "uplo": uplo, "flb": flb,
               "gen": name.split("_")[0], "x_ref_norm": float(np.linalg.norm(x)),
               "x_ref_err_vs_true": float(np.linalg.norm(x - x_true) / np.linalg.norm(x_true)),
               "arrays": {k: digest(v) for k, v in st.items() if isinstance(v, np.ndarray)},
               "sizes": {k: int(v.size) for k, v in st.items() if isinstance(v, np.ndarray)},
               "scalars": {k: int(v) for k, v in st.items() if not isinstance(v, np.ndarray)}}
        dig[name] = rec
        print(name, rec["scalars"])
    with open(os.path.join(HERE, "digest.json"), "w") as f:
        json.dump(dig, f, indent=1, sort_keys=True)


def full_cases():
    """The banded workload at full size (m = 4,194,304): 'L' and 'U' (the
    transpose) at every swept partition count."""
    L = synth.banded_lower(4194304, seed=0)
    out = [(f"banded4194304_L_P{P}", L, P, "L", 1) for P in (16, 64, 256, 1024)]
    U = synth.transpose(L)
    out += [(f"banded4194304_U_P{P}", U, P, "U", 1) for P in (16, 64, 256, 1024)]
    return out


def x_sample_index(m: int) -> np.ndarray:
    """Rows whose x values are stored for the full-size cases: every 997th row plus
    the first and last 64 (where the mirror and the partition edges meet)."""
    idx = np.concatenate([np.arange(0, m, 997), np.arange(64), np.arange(m - 64, m)])
    return np.unique(idx)


def main_full():
    """Digests of every structure array for the full-size banded cases, merged into
    digest.json, and the reference's x at sampled rows (full_x_samples.npz)."""
    if not oracle.Reference.available():
        raise SystemExit("oracle/_ref/libspike_ref.so is missing: make -C oracle ref")
    path = os.path.join(HERE, "digest.json")
    with open(path) as f:
        dig = json.load(f)
    spath = os.path.join(HERE, "full_x_samples.npz")
    samples = dict(np.load(spath)) if os.path.exists(spath) else {}
    for name, A, P, uplo, flb in full_cases():
        x_true, b = synth.make_rhs(A, seed=0)
        st, x = run_reference(A, P, uplo, flb, b)
        rec = {"m": int(A.m), "nnz": int(A.nnz), "P": P, "uplo": uplo, "flb": flb,
               "gen": name.split("_")[0], "x_ref_norm": float(np.linalg.norm(x)),
               "x_ref_err_vs_true": float(np.linalg.norm(x - x_true) / np.linalg.norm(x_true)),
               "arrays": {k: digest(v) for k, v in st.items() if isinstance(v, np.ndarray)},
               "sizes": {k: int(v.size) for k, v in st.items() if isinstance(v, np.ndarray)},
               "scalars": {k: int(v) for k, v in st.items() if not isinstance(v, np.ndarray)}}
        dig[name] = rec
        samples[name] = x[x_sample_index(A.m)]
        print(name, rec["scalars"], "err vs x_true", rec["x_ref_err_vs_true"], flush=True)
        with open(path, "w") as f:
            json.dump(dig, f, indent=1, sort_keys=True)
        np.savez_compressed(spath, **samples)


if __name__ == "__main__":
    if "--full" in sys.argv:
        main_full()
    else:
        main()
