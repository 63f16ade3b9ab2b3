"""Serving loop: requests of uneven size, order, final time and limiter
setting run together in one device pool; each result equals the same solve
run alone through the server and through a single-solve context (bit for
bit), admission respects the HBM budget and the slot count, and a request
that goes non-physical fails alone."""
import math
import time

import numpy as np
import pytest

from rkdg_heter_calculate_b200 import CUDARkdgSolver, capi, meshgen, vortex
from rkdg_heter_calculate_b200.serve import DONE, Server
from rkdg_heter_calculate_b200.solver import freestream_state, primitive_to_conservative

pytestmark = pytest.mark.gpu
MB = 1 << 20
# Each request carries its flux: HLLC for the vortex requests, LLF for the
# limited ones (the Mach-3 step with the Davis-speed HLLC flux goes
# non-physical at the step corner, FP64 and FP32 alike, under P1 + TVB)
TVB_M = 50.0
SERVER = dict(flux="llf", rk=3, cfl=0.2, tvb_m=TVB_M)


def requests():
    """(mesh, order, U0 native, t_final, far field, limiter, flux): vortex
    requests with HLLC, the limited ones with LLF."""
    out = []
    for m, order, beta, th, tf in [
        (meshgen.periodic_delaunay(20, seed=11), 2, 5.0, 0.3, 0.21),
        (meshgen.periodic_structured(14, 14, jitter=0.2, seed=12), 1, 3.0, 1.2, 0.35),
        (meshgen.periodic_delaunay(12, seed=13), 2, 2.0, 4.0, 0.08),
        (meshgen.periodic_delaunay(9, seed=14), 1, 1.5, 2.5, 0.5),
    ]:
        ui, vi = math.sqrt(2) * math.cos(th), math.sqrt(2) * math.sin(th)
        nb = 3 if order == 1 else 6
        U = vortex.project_native(m, lambda X, Y: vortex.exact(X, Y, 0.0, beta, 1.4, ui, vi), nb)
        far = np.array([1.0, ui, vi, 2.5 + 0.5 * (ui * ui + vi * vi)])
        out.append((m, order, U, tf, far, False, "hllc"))
    # Mach-3 wind-tunnel step, P1 with the TVB limiter, started from the inflow state
    step = meshgen.forward_step(h=1.0 / 30)
    far = np.array(primitive_to_conservative(1.4, 3.0, 0.0, 1.0))
    U = np.zeros((4, 3, step.ntri))
    U[:, 0, :] = far[:, None]
    out.append((step, 1, U, 0.02, far, True, "llf"))
    # subsonic flow around a square cylinder, P2 with the limiter
    box = meshgen.box_with_obstacle(16)
    far = np.array(freestream_state())
    U = np.zeros((4, 6, box.ntri))
    U[:, 0, :] = far[:, None]
    out.append((box, 2, U, 1.0, far, True, "llf"))
    return out


def solo(req, precision):
    m, order, U, tf, far, lim, flux = req
    kw = dict(order=2, nq=6, ng=3) if order == 2 else dict(order=1, nq=3, ng=2)
    s = CUDARkdgSolver(m, flux=flux, rk=3, precision=precision, cfl=0.2, farfield=far,
                       limiter="tvb" if lim else None, tvb_m=TVB_M, **kw)
    s.setFreedom(U, basis="native")
    t, n = s.advance(1000000, t_final=tf)
    out = s.copyFreedomToHost(basis="native")
    s.close()
    return out, t, n


def submit(srv, req):
    m, order, U, tf, far, lim, flux = req
    return srv.submit(m, order, U, tf, farfield=far, limiter=lim, flux=flux)


@pytest.mark.parametrize("precision", ["fp32", "fp32c", "fp64"])
def test_results_same_alone_and_in_the_mix(precision):
    reqs = requests()
    with Server(256 * MB, max_slots=8, precision=precision, **SERVER) as srv:
        alone = []
        for r in reqs:
            res = srv.wait(submit(srv, r))
            assert res.status == DONE
            alone.append(res)
        # staggered arrivals: half now, the rest while those run
        ids = [submit(srv, r) for r in reqs[::2]]
        time.sleep(0.02)
        ids += [submit(srv, r) for r in reqs[1::2]]
        order = list(range(0, len(reqs), 2)) + list(range(1, len(reqs), 2))
        mixed = {i: srv.wait(rid) for i, rid in zip(order, ids)}
        st = srv.stats()
    assert st["completed"] == 2 * len(reqs)
    assert st["peak_in_flight"] >= 2
    for i, r in enumerate(reqs):
        ref, t, n = solo(r, precision)
        assert n == alone[i].steps == mixed[i].steps, f"request {i}"
        np.testing.assert_array_equal(alone[i].state, ref, err_msg=f"request {i} alone")
        np.testing.assert_array_equal(mixed[i].state, ref, err_msg=f"request {i} in the mix")
        assert mixed[i].submitted <= mixed[i].admitted <= mixed[i].completed


def test_budget_and_slots_bound_admission():
    reqs = requests()
    big = max(r[0].ntri for r in reqs)
    # a pool of about 1.2x the largest request: the rest queue until memory frees
    per_elem = 3 * 24 * 4 + 108 + 192   # FP32 pool bytes per element, staging included
    budget = 64 * MB + int(1.2 * big) * per_elem
    with Server(budget, max_slots=3, precision="fp32", **SERVER) as srv:
        cap = srv.stats()["capacity_elements"]
        assert big <= cap < sum(r[0].ntri for r in reqs)
        ids = [submit(srv, r) for r in reqs]
        res = [srv.wait(i) for i in ids]
        st = srv.stats()
    assert all(r.status == DONE for r in res)
    assert 1 <= st["peak_in_flight"] <= 3
    for r, q in zip(res, reqs):
        ref, _, n = solo(q, "fp32")
        assert r.steps == n
        np.testing.assert_array_equal(r.state, ref)


def test_oversized_request_rejected():
    reqs = requests()
    per_elem = 3 * 24 * 4 + 108 + 192   # FP32 pool bytes per element, staging included
    with Server(64 * MB + 4300 * per_elem, max_slots=2, precision="fp32", **SERVER) as srv:
        step = reqs[4]
        assert step[0].ntri > srv.stats()["capacity_elements"]
        with pytest.raises(capi.RkdgError) as e:
            submit(srv, step)
        assert e.value.code == capi.RKDG_ERR_NOMEM


def test_failed_request_fails_alone():
    reqs = requests()
    m, order, U, tf, far, lim, flux = reqs[2]
    bad = U.copy()
    bad[0, 0, 5] = -1.0   # negative density in one cell
    with Server(128 * MB, max_slots=4, precision="fp32", **SERVER) as srv:
        good_id = submit(srv, reqs[3])
        bad_id = srv.submit(m, order, bad, tf, farfield=far, flux=flux)
        with pytest.raises(capi.RkdgError) as e:
            srv.wait(bad_id)
        assert e.value.code == capi.RKDG_ERR_STATE
        res = srv.wait(good_id)
    assert res.status == DONE
    ref, _, _ = solo(reqs[3], "fp32")
    np.testing.assert_array_equal(res.state, ref)


def test_engine_failure_fails_every_request_and_is_reported():
    """A failure of the loop (a CUDA call failing, simulated on the host by
    rkdg_server_inject_fault: nothing touches the device) fails every request
    that is in flight or queued, is reported by the status query, and later
    submits are refused."""
    reqs = requests()
    with Server(256 * MB, max_slots=2, precision="fp32", **SERVER) as srv:
        assert srv.status() == {"queued": 0, "in_flight": 0}
        long_run = (reqs[0][0], reqs[0][1], reqs[0][2], 50.0, reqs[0][4], False, "hllc")
        ids = [submit(srv, long_run) for _ in range(4)]  # two in flight, two queued (2 slots)
        time.sleep(0.2)
        st = srv.status()
        assert st["in_flight"] == 2 and st["queued"] == 2
        srv.inject_fault(1)
        for rid in ids:
            with pytest.raises(capi.RkdgError) as e:
                srv.wait(rid, timeout=60.0)
            assert e.value.code == capi.RKDG_ERR_CUDA and "inject_fault" in str(e.value)
        with pytest.raises(capi.RkdgError) as e:
            srv.status()
        assert e.value.code == capi.RKDG_ERR_CUDA
        with pytest.raises(capi.RkdgError) as e:
            submit(srv, reqs[3])
        assert e.value.code == capi.RKDG_ERR_CUDA
