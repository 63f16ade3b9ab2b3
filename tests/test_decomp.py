"""Domain decomposition on the host: the partition's lists, and the
decomposed time loop (halo exchange before every stage, dt as the minimum
over parts, halo means refreshed before the limiter) against the
single-domain run.

The per-part compute here is the oracle (test infrastructure, CPU), driven
through the same DecomposedSolve loop and transports the device path uses:
LocalTransport with three parts in one process, and TorchTransport with two
gloo ranks.  Each owned element sees exact copies of its neighbours, so the
decomposed result equals the single-domain oracle run bit for bit."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from helpers import project_reference, vortex_state
from oracle import oracle
from rkdg_heter_calculate_b200 import meshgen
from rkdg_heter_calculate_b200.decomp import DecomposedSolve, LocalTransport, Partition, TorchTransport
from rkdg_heter_calculate_b200.solver import primitive_to_conservative

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TESTS = os.path.dirname(os.path.abspath(__file__))


class OraclePart:
    """One part computed by the oracle: the DevicePart interface on host
    arrays (rows are basis rows of the reference-basis state)."""

    def __init__(self, partition, p, limiter, **kw):
        import torch

        self.torch = torch
        self.n_owned = partition.n_owned(p)
        self.o = oracle.Oracle(partition.local_mesh(p), limiter=oracle.LIMITER_NONE, **kw)
        self.send = {q: v for q, v in partition.send[p].items()}
        self.recv = {q: v for q, v in partition.recv[p].items()}
        self.nb = self.o.nb

    def set_state(self, U):
        self.o.set_state(U)

    def state(self):
        return self.o.state()

    def time_step(self):
        return self.o.time_step()

    def save_old(self):
        self.o.save_old()

    def stage(self, st, dt):
        self.o.stage(st, dt)

    def limit(self):
        self.o.limit()

    def buffer(self, q, incoming, means_only):
        n = (self.recv if incoming else self.send)[q].size
        return self.torch.empty((4, 1 if means_only else self.nb, n), dtype=self.torch.float64)

    def pack(self, q, means_only):
        k = 1 if means_only else self.nb
        return self.torch.from_numpy(np.ascontiguousarray(self.o.state()[:, :k, self.send[q]]))

    def unpack(self, q, means_only, buf):
        k = 1 if means_only else self.nb
        U = self.o.state()
        U[:, :k, self.recv[q]] = buf.numpy()
        self.o.set_state(U)

    def sync(self):
        pass


def case(kind):
    if kind == "vortex":
        mesh = meshgen.periodic_delaunay(16, seed=4)
        far = primitive_to_conservative(1.0, 1.0, 1.0, 1.0)
        kw = dict(order=2, nq=6, ng=3, flux=oracle.HLLC, rk=3, farfield=far, cfl=0.2)
        o = oracle.Oracle(mesh, **kw)
        U0 = vortex_state(mesh, o.basis()["coeff"], 6)
        return mesh, kw, False, U0
    mesh = meshgen.channel(30, 10, jitter=0.2, seed=8)
    far = primitive_to_conservative(1.4, 3.0, 0.0, 1.0)
    kw = dict(order=1, nq=3, ng=2, flux=oracle.LLF, rk=3, farfield=far, cfl=0.3, tvb_m=50.0)
    o = oracle.Oracle(mesh, **kw)

    def shock(X, Y):
        left = X + 0.2 * Y < 1.2
        return np.stack(primitive_to_conservative(np.where(left, 1.4, 3.0), np.where(left, 3.0, 1.2),
                                                  0 * X, np.where(left, 1.0, 4.0)))

    return mesh, kw, True, project_reference(mesh, shock, o.basis()["coeff"], 3)


def single_domain(mesh, kw, limiter, U0, nsteps):
    o = oracle.Oracle(mesh, limiter=oracle.LIMITER_TVB if limiter else oracle.LIMITER_NONE, **kw)
    o.set_state(U0)
    dts = [o.step()[0] for _ in range(nsteps)]
    return o.state(), dts


def test_partition_lists():
    mesh = meshgen.periodic_delaunay(20, seed=2)
    P = Partition(mesh, 4)
    assert sorted(np.concatenate(P.owned).tolist()) == list(range(mesh.ntri))
    for p in range(4):
        lm = P.local_mesh(p)
        lm.check()
        n = P.n_owned(p)
        assert (lm.neighbours[:n] >= 0).all()  # periodic: every owned edge has a local neighbour
        assert set(P.halo[p]) & set(P.owned[p]) == set()
        for q, r in P.recv[p].items():
            s = P.send[q][p]
            assert r.size == s.size
            # the rows q sends are the elements p holds as halo copies, in order
            np.testing.assert_array_equal(P.owned[q][s], P.local_ids(p)[r])


@pytest.mark.parametrize("kind", ["vortex", "step"])
def test_three_parts_in_one_process_equal_single_domain(kind):
    mesh, kw, limiter, U0 = case(kind)
    ref, dts = single_domain(mesh, kw, limiter, U0, 6)
    P = Partition(mesh, 3)
    parts = {p: OraclePart(P, p, limiter, **kw) for p in range(3)}
    for p, part in parts.items():
        part.set_state(P.split(U0, p))
    solve = DecomposedSolve(parts, LocalTransport(), rk=kw["rk"], limiter=limiter)
    got_dts = [solve.step() for _ in range(6)]
    assert got_dts == dts
    np.testing.assert_array_equal(P.join({p: part.state() for p, part in parts.items()}), ref)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, kind, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    for path in (ROOT, TESTS):
        sys.path.insert(0, path)
    import datetime

    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mesh, kw, limiter, U0 = case(kind)
        P = Partition(mesh, world)
        part = OraclePart(P, rank, limiter, **kw)
        part.set_state(P.split(U0, rank))
        solve = DecomposedSolve({rank: part}, TorchTransport(), rk=kw["rk"], limiter=limiter)
        dts = [solve.step() for _ in range(6)]
        q.put((rank, dts, part.state()[:, :, : P.n_owned(rank)]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("kind", ["vortex", "step"])
def test_two_gloo_ranks_equal_single_domain(kind):
    mesh, kw, limiter, U0 = case(kind)
    ref, dts = single_domain(mesh, kw, limiter, U0, 6)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, kind, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(2):
        rank, got_dts, U = q.get(timeout=180)
        out[rank] = U
        assert got_dts == dts
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    P = Partition(mesh, 2)
    np.testing.assert_array_equal(P.join(out), ref)
