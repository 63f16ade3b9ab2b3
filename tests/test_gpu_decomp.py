"""Domain decomposition on the device: three partition contexts
(rkdg_create_part) on one GPU, their halo rows moved by rkdg_gather_rows /
rkdg_scatter_rows before every stage, dt the minimum over the parts and,
with the limiter, the halo means refreshed before rkdg_limit.  The
decomposed run matches the oracle and the single-context run to 1e-12 in
FP64 (each part tiles its own elements, so interface fluxes are formed from
the other side than in the single context: equal to rounding, not bit for
bit), and the FP32C form stays within FP32 rounding of its single-context
run.  The stream-ordered loop (DecomposedSolve.advance_device: halo
transfers, the wave-speed all-reduce and the stages enqueued with no host
round trip) equals the host-driven loop and lands on a final time like the
single context.  Between GPUs the same loops move the rows with NCCL
(decomp.TorchTransport); the host tests cover that transport with gloo."""
import ctypes as C

import numpy as np
import pytest
import torch

from helpers import rel_err
from oracle import oracle
from rkdg_heter_calculate_b200 import CUDARkdgSolver, capi
from rkdg_heter_calculate_b200.decomp import DecomposedSolve, DevicePart, LocalTransport, Partition
from test_decomp import case, single_domain

pytestmark = pytest.mark.gpu
NSTEPS = 6


def solver_kw(kw, limiter, precision):
    return dict(order=kw["order"], nq=kw["nq"], ng=kw["ng"], flux="hllc" if kw["flux"] == oracle.HLLC else "llf",
                rk=kw["rk"], cfl=kw["cfl"], farfield=kw["farfield"], limiter="tvb" if limiter else None,
                tvb_m=kw.get("tvb_m", 50.0), precision=precision)


def decomposed(mesh, kw, limiter, U0, precision, nparts=3, device_loop=False, t_final=0.0, graph=False,
               overlap=None):
    P = Partition(mesh, nparts)
    parts = {p: DevicePart(P, p, **solver_kw(kw, limiter, precision)) for p in range(nparts)}
    for p, part in parts.items():
        part.set_state(P.split(U0, p))
    solve = DecomposedSolve(parts, LocalTransport(), rk=kw["rk"], limiter=limiter, overlap=overlap)
    if device_loop:
        dts = solve.advance_device(NSTEPS if t_final <= 0 else 10 ** 6, t_final=t_final, graph=graph)  # (t, steps)
    else:
        dts = [solve.step() for _ in range(NSTEPS)]
    U = P.join({p: part.state() for p, part in parts.items()})
    for part in parts.values():
        part.close()
    return U, dts


def single_context(mesh, kw, limiter, U0, precision):
    s = CUDARkdgSolver(mesh, **solver_kw(kw, limiter, precision))
    s.setFreedom(U0)
    dts = [s.step()[0] for _ in range(NSTEPS)]
    U = s.copyFreedomToHost()
    s.close()
    return U, dts


@pytest.mark.parametrize("kind", ["vortex", "step"])
def test_device_parts_match_oracle_and_single_context(kind):
    mesh, kw, limiter, U0 = case(kind)
    ref, ref_dts = single_domain(mesh, kw, limiter, U0, NSTEPS)
    U, dts = decomposed(mesh, kw, limiter, U0, "fp64")
    np.testing.assert_allclose(dts, ref_dts, rtol=1e-12)
    assert rel_err(U, ref) < 1e-12
    one, _ = single_context(mesh, kw, limiter, U0, "fp64")
    assert rel_err(U, one) < 1e-12


@pytest.mark.parametrize("kind,overlap", [("vortex", False), ("step", False), ("vortex", True), ("step", True)])
def test_device_loop_equals_host_loop(kind, overlap):
    """advance_device (no host round trip per step; with overlap, each
    stage's halo transfers beside its interior tiles) against the
    host-driven step loop: the same time and the same states (FP64)."""
    mesh, kw, limiter, U0 = case(kind)
    host, dts = decomposed(mesh, kw, limiter, U0, "fp64")
    dev, (t, n) = decomposed(mesh, kw, limiter, U0, "fp64", device_loop=True, overlap=overlap)
    assert n == NSTEPS
    assert t == pytest.approx(sum(dts), rel=1e-13)
    assert rel_err(dev, host) < 1e-12


@pytest.mark.parametrize("kind,overlap", [("vortex", False), ("step", False), ("step", True)])
def test_graph_replay_equals_device_loop(kind, overlap):
    """One decomposed step captured as a CUDA graph and replayed: the same
    bits as the enqueued loop."""
    mesh, kw, limiter, U0 = case(kind)
    a, (ta, na) = decomposed(mesh, kw, limiter, U0, "fp32", device_loop=True, overlap=overlap)
    b, (tb, nb) = decomposed(mesh, kw, limiter, U0, "fp32", device_loop=True, graph=True, overlap=overlap)
    assert (ta, na) == (tb, nb)
    np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("kind", ["vortex", "step"])
def test_split_stage_equals_whole_stage(kind):
    """rkdg_part_stage_begin + rkdg_part_stage_end (the tiles that read no
    halo copy, then the rest) give the bits of rkdg_part_stage."""
    mesh, kw, limiter, U0 = case(kind)
    P = Partition(mesh, 3)
    out = []
    for split in (False, True):
        parts = {p: DevicePart(P, p, **solver_kw(kw, limiter, "fp64")) for p in range(3)}
        for p, part in parts.items():
            part.set_state(P.split(U0, p))
        tr = LocalTransport()
        bufs = {p: torch.zeros(1, dtype=torch.float64, device="cuda") for p in parts}
        for _ in range(2):
            tr.exchange(parts, False)
            for p, part in parts.items():
                part.wave_out(bufs[p])
            tr.max_device(parts, bufs)
            for p, part in parts.items():
                part.wave_in(bufs[p])
                part.begin_step()
            for st in range(kw["rk"]):
                if st > 0:
                    tr.exchange(parts, False)
                for part in parts.values():
                    if split:
                        part.stage_begin(st)
                        part.stage_end(st)
                    else:
                        part.stage_async(st)
                if limiter:
                    tr.exchange(parts, True)
                    for part in parts.values():
                        part.limit_async()
        out.append(P.join({p: part.state() for p, part in parts.items()}))
        for part in parts.values():
            part.close()
    np.testing.assert_array_equal(out[0], out[1])


def test_device_loop_lands_on_final_time():
    mesh, kw, limiter, U0 = case("vortex")
    one = CUDARkdgSolver(mesh, **solver_kw(kw, limiter, "fp32"))
    one.setFreedom(U0)
    t1, n1 = one.advance(10 ** 6, t_final=0.05)
    ref = one.copyFreedomToHost()
    one.close()
    dev, (t, n) = decomposed(mesh, kw, limiter, U0, "fp32", device_loop=True, t_final=0.05)
    assert t == t1 == 0.05 and n == n1
    assert rel_err(dev, ref) < 1e-5


def test_fp32c_parts_track_single_context():
    mesh, kw, limiter, U0 = case("vortex")
    U, _ = decomposed(mesh, kw, limiter, U0, "fp32c")
    one, _ = single_context(mesh, kw, limiter, U0, "fp32c")
    assert rel_err(U, one) < 1e-5


def test_bad_halo_index_is_reported():
    """An index outside the partition is skipped by the exchange kernel and
    reported at the next sync (no out-of-range access)."""
    mesh, kw, limiter, U0 = case("vortex")
    P = Partition(mesh, 2)
    part = DevicePart(P, 0, **solver_kw(kw, limiter, "fp64"))
    part.set_state(P.split(U0, 0))
    idx = torch.tensor([0, 10 ** 7], dtype=torch.int32, device="cuda")
    buf = torch.empty((2, part.rows[False], 16), dtype=torch.uint8, device="cuda")
    lib = capi.lib()
    assert lib.rkdg_gather_rows(part.s.h, C.c_void_p(idx.data_ptr()), 2, part.rows[False],
                                C.c_void_p(buf.data_ptr())) == capi.RKDG_OK
    with pytest.raises(capi.RkdgError) as e:
        part.sync()
    assert e.value.code == capi.RKDG_ERR_INVALID
    part.close()
