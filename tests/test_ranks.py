"""The multi-GPU replica rules of bench.py on CPU: world_size-2 gloo ranks agree
on the slowest rank's time and the whole-job value; the reference arm runs on
rank 0 only."""
import os
import socket

import pytest
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ms = [3.0, 5.0][rank]
    m = bench.max_over_ranks(ms, "cpu", world)
    out[rank] = (m, bench.replicas_value(m, world))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_slowest_time():
    ctx = mp.get_context("spawn")
    port = _free_port()
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        got = dict(out)
    assert got[0] == got[1] == (5.0, 2 * 1e3 / 5.0)


def test_single_rank_needs_no_collective():
    assert bench.max_over_ranks(4.0, "cpu", 1) == 4.0
    assert bench.replicas_value(4.0, 1) == 250.0


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    monkeypatch.setenv("RANK", "1")

    class A:
        P = 1024
        steps = 1
        warmup = 3
    assert bench.run_reference(A()) == 0
    assert capsys.readouterr().out == ""
