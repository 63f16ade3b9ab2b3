"""Known-answer tests of the oracle's extensions beyond the reference
(P1, 3/6-point and 2-point rules, HLLC, SSP-RK2, TVB limiter), which have
no reference code to be pinned against."""
import numpy as np
import pytest

from helpers import perturbed_state, project_reference, vortex_state
from oracle import oracle
from rkdg_heter_calculate_b200 import meshgen, vortex
from rkdg_heter_calculate_b200.solver import primitive_to_conservative

CONFIGS = [
    dict(order=2, nq=7, ng=3, flux=oracle.LLF, rk=3),
    dict(order=2, nq=6, ng=3, flux=oracle.HLLC, rk=3),
    dict(order=1, nq=3, ng=2, flux=oracle.LLF, rk=2),
    dict(order=1, nq=3, ng=2, flux=oracle.HLLC, rk=3),
]


@pytest.mark.parametrize("cfg", CONFIGS)
def test_free_stream_is_preserved(cfg):
    mesh = meshgen.periodic_structured(6, 5, jitter=0.25, seed=4)
    far = primitive_to_conservative(1.2, 0.7, -0.4, 0.9)
    o = oracle.Oracle(mesh, farfield=far, **cfg)
    U = np.zeros((4, o.nb, mesh.ntri))
    U[:, 0, :] = np.array(far)[:, None]
    o.set_state(U)
    R = o.residual()
    assert np.abs(R).max() < 1e-13
    o.step()
    assert np.abs(o.state() - U).max() < 1e-13


@pytest.mark.parametrize("cfg", CONFIGS)
def test_periodic_conservation(cfg):
    mesh = meshgen.periodic_structured(6, 6, jitter=0.2, seed=9)
    o = oracle.Oracle(mesh, **cfg)
    U = vortex_state(mesh, o.basis()["coeff"], o.nb, beta=4.0)
    o.set_state(U)
    area = mesh.areas()
    tot0 = (o.state()[:, 0, :] * area).sum(axis=1)
    for _ in range(5):
        o.step()
    tot = (o.state()[:, 0, :] * area).sum(axis=1)
    np.testing.assert_allclose(tot, tot0, rtol=1e-13, atol=1e-13)


def test_hllc_resolves_stationary_contact():
    # a density jump with equal pressure and zero velocity is an exact
    # stationary contact: HLLC keeps it, LLF diffuses it
    mesh = meshgen.channel(12, 4, jitter=0.0)
    c = mesh.coords().mean(axis=1)

    def state(X, Y):
        rho = np.where(X < 1.5, 1.0, 0.25) * np.ones_like(X)
        return np.stack(primitive_to_conservative(rho, 0 * X, 0 * X, 1.0 + 0 * X))

    res = {}
    for flux in (oracle.HLLC, oracle.LLF):
        o = oracle.Oracle(mesh, order=1, nq=3, ng=2, flux=flux, rk=3,
                          farfield=primitive_to_conservative(1.0, 0.0, 0.0, 1.0))
        U = np.zeros((4, 3, mesh.ntri))
        U[:, 0, :] = state(c[:, 0], c[:, 1])
        o.set_state(U)
        res[flux] = np.abs(o.residual()[0]).max()
    # cells whose centroid lies in the interior column pair across x = 1.5
    assert res[oracle.HLLC] < 1e-12
    assert res[oracle.LLF] > 1e-3


def test_tvb_limiter_keeps_linear_data_and_smooth_data():
    mesh = meshgen.channel(16, 6, jitter=0.2, seed=2)
    far = primitive_to_conservative(1.0, 0.5, 0.0, 1.0)
    o = oracle.Oracle(mesh, order=1, nq=3, ng=2, limiter=oracle.LIMITER_TVB, tvb_m=0.0,
                      farfield=far)
    coeff = o.basis()["coeff"]

    def lin(X, Y):
        r = 1.0 + 0.05 * X + 0.03 * Y
        return np.stack(primitive_to_conservative(r, 0.5 + 0 * X, 0 * X, 1.0 + 0.02 * X))

    U = project_reference(mesh, lin, coeff, 3)
    o.set_state(U)
    o.limit()
    V = o.state()
    interior = (mesh.neighbours >= 0).all(axis=1)
    # second ring: all neighbours interior too
    ring2 = interior & interior[np.maximum(mesh.neighbours, 0)].all(axis=1)
    assert np.abs(V[:, :, ring2] - U[:, :, ring2]).max() < 1e-12
    # with a huge M nothing is limited at all
    o2 = oracle.Oracle(mesh, order=1, nq=3, ng=2, limiter=oracle.LIMITER_TVB, tvb_m=1e12,
                       farfield=far)
    W = perturbed_state(mesh, coeff, 3, far, amp=0.2)
    o2.set_state(W)
    assert o2.limit() == 0
    assert np.abs(o2.state() - W).max() == 0.0


def test_tvb_limiter_limits_a_discontinuity_and_conserves():
    # fine enough that M h^2 (M = 50) is far below the jump
    mesh = meshgen.channel(60, 20, jitter=0.2, seed=2)
    far = primitive_to_conservative(1.0, 0.0, 0.0, 1.0)
    o = oracle.Oracle(mesh, order=1, nq=3, ng=2, limiter=oracle.LIMITER_TVB, tvb_m=50.0,
                      farfield=far)
    coeff = o.basis()["coeff"]

    def step(X, Y):
        r = np.where(X + 0.3 * Y < 1.4, 1.0, 0.125)
        p = np.where(X + 0.3 * Y < 1.4, 1.0, 0.1)
        return np.stack(primitive_to_conservative(r, 0 * X, 0 * X, p))

    U = project_reference(mesh, step, coeff, 3)
    o.set_state(U)
    n = o.limit()
    V = o.state()
    assert n > 0
    np.testing.assert_array_equal(V[:, 0, :], U[:, 0, :])  # means untouched
    # limited slopes do not exceed the unlimited ones near the jump
    assert np.abs(V[0, 1:]).max() <= np.abs(U[0, 1:]).max() + 1e-14


def test_vortex_error_decreases_with_order_of_accuracy():
    errs = []
    for n in (8, 16):
        mesh = meshgen.periodic_structured(n, n, jitter=0.0)
        o = oracle.Oracle(mesh, order=1, nq=3, ng=2, rk=3, cfl=0.3)
        U = vortex_state(mesh, o.basis()["coeff"], 3)
        o.set_state(U)
        t = 0.0
        while t < 0.5 - 1e-12:
            dt = min(o.time_step(), 0.5 - t)
            o.step(dt)
            t += dt
        # evaluate at element quadrature points
        xi, eta, w = vortex.triangle_rule(5)
        X, Y = vortex.physical_points(mesh, xi, eta)
        uh = o.eval(xi, eta)[0].T
        ex = vortex.exact(X, Y, 0.5)[0]
        area = mesh.areas()
        errs.append(np.sqrt((area[:, None] * w[None] * (uh - ex) ** 2).sum() / area.sum()))
    rate = np.log2(errs[0] / errs[1])
    assert rate > 1.5, errs
