"""The bench's multi-rank path on CPU: two gloo ranks launched as torchrun
would (RANK / WORLD_SIZE / MASTER_* in the environment).  Every rank runs
the same collectives in the same order; times reduce by max over ranks and
units by sum, so the whole-job rate is the units of all ranks over the
slowest rank's time.  The reference arm runs on rank 0 only; other ranks
return without work or output."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench

    d = bench.Dist(backend="gloo")
    d.init()
    try:
        d.barrier()
        t_max = d.max(10.0 + rank)          # per-rank time (ms): the slowest counts
        units = d.sum(1000.0 * (rank + 1))   # per-rank units: all count
        rate = units / (t_max * 1e-3)
        d.barrier()
        q.put((rank, t_max, units, rate))
    finally:
        d.close()


def test_two_gloo_ranks_reduce_like_the_bench():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=10) for _ in range(2))
    for rank, t_max, units, rate in out:
        assert t_max == 11.0
        assert units == 3000.0
        assert rate == pytest.approx(3000.0 / 11e-3)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    sys.path.insert(0, ROOT)
    import bench

    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--gpus", "2"])
    called = []
    monkeypatch.setattr(bench, "cpu_reference_sample", lambda *a, **k: called.append(1))
    bench.main()
    assert not called
    assert capsys.readouterr().out == ""
