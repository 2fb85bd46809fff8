"""The sharded chain solve on CPU: world_size 2 and 3 gloo ranks, each running
its shard's phases with the CPU restatement of the chain solve (chain_ref.py),
exchanging the halo rows point to point; the assembled x must match the
sequential substitution within 1e-12, for uplo 'L' and 'U'."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _case(uplo):
    from spike_pstrsv_b200 import synth

    L = synth.banded_lower(16384, seed=21)
    A = L if uplo == "L" else synth.transpose(L)
    x_true, b = synth.make_rhs(A, seed=21)
    return A, b


def _rank(rank, world, port, uplo, plan, out):
    import sys

    sys.path.insert(0, HERE)
    sys.path.insert(0, os.path.dirname(HERE))
    import torch
    import torch.distributed as dist

    import chain_ref
    from spike_pstrsv_b200 import shard

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    A, b = _case(uplo)
    U, rev = chain_ref.upper(A, uplo)
    tasks, reach = plan
    S = shard.ShardedSolve(chain_ref.NumpyBackend(U, rev, tasks), A.m, uplo, reach, tasks, rank, world)
    tb = torch.from_numpy(b)
    tx = torch.full((A.m,), float("nan"), dtype=torch.float64)  # rows no rank writes stay NaN
    S.solve(tb, tx)
    out[rank] = (S.rows().start, S.rows().stop, tx[S.rows()].numpy().copy(), reach)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("uplo", ["L", "U"])
def test_sharded_chain_solve_matches_substitution(world, uplo):
    import sys

    import oracle

    sys.path.insert(0, HERE)
    import chain_ref

    A, b = _case(uplo)
    plan = chain_ref.chain_plan(chain_ref.upper(A, uplo)[0], 2048)  # once, shared by the ranks
    ctx = mp.get_context("spawn")
    port = _free_port()
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_rank, args=(r, world, port, uplo, plan, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(300)
            assert p.exitcode == 0
        x = np.full(A.m, np.nan)
        covered = 0
        for r in range(world):
            lo, hi, part, _ = out[r]
            x[lo:hi] = part
            covered += hi - lo
    assert covered == A.m and np.isfinite(x).all()
    xs = oracle.sequential_solve(A, b, uplo)
    assert np.linalg.norm(x - xs) <= 1e-12 * np.linalg.norm(xs)


def test_plan_splits_whole_chains():
    from spike_pstrsv_b200 import shard

    tasks = np.array([(a, min(a + 100, 950), a, min(a + 100, 950)) for a in range(0, 950, 100)]).reshape(-1)
    for world in (1, 2, 3, 10):
        ranges = shard.plan(tasks, world)
        assert ranges[0][0] == 0 and ranges[-1][1] == 950
        assert all(ranges[r][1] == ranges[r + 1][0] for r in range(world - 1))
        assert all(lo % 100 == 0 and lo < hi for lo, hi in ranges)
    with pytest.raises(ValueError):
        shard.plan(tasks, 11)
