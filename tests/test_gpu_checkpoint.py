"""Checkpoint and resume: a run stopped after some steps, written to a file
and restored into a fresh context on the same mesh continues bit for bit
(state, time and step count) as the run that never stopped; a file written
for another mesh, order, precision, far field, flux, CFL number or gamma is
refused, and a missing file is an I/O error."""
import numpy as np
import pytest

from rkdg_heter_calculate_b200 import CUDARkdgSolver, capi, meshgen, vortex
from rkdg_heter_calculate_b200.solver import primitive_to_conservative

pytestmark = pytest.mark.gpu
FAR = primitive_to_conservative(1.0, 1.0, 1.0, 1.0)


def solver(mesh, precision, order=2, limiter=None, far=FAR):
    kw = dict(order=2, nq=6, ng=3) if order == 2 else dict(order=1, nq=3, ng=2)
    return CUDARkdgSolver(mesh, flux="hllc", rk=3, precision=precision, cfl=0.2, farfield=far,
                          limiter=limiter, **kw)


@pytest.mark.parametrize("precision", ["fp32", "fp32c", "fp64"])
@pytest.mark.parametrize("order", [1, 2])
def test_resume_is_bitwise(tmp_path, precision, order):
    mesh = meshgen.periodic_delaunay(16, seed=5)
    nb = 3 if order == 1 else 6
    U0 = vortex.project_native(mesh, lambda X, Y: vortex.exact(X, Y, 0.0), nb)
    path = str(tmp_path / "run.ckpt")
    a = solver(mesh, precision, order)
    a.setFreedom(U0, basis="native")
    a.advance(7)
    a.checkpoint(path)
    t_a, n_a = a.advance(5)
    ref = a.copyFreedomToHost(basis="native")
    t_ref, steps_ref = a.time()
    a.close()
    b = solver(mesh, precision, order)
    b.restore(path)
    t_b, n_b = b.advance(5)
    assert n_b == n_a == 5 and t_b == t_ref
    assert b.time() == (t_ref, steps_ref)
    np.testing.assert_array_equal(b.copyFreedomToHost(basis="native"), ref)
    b.close()


def test_resume_with_final_time_and_limiter(tmp_path):
    mesh = meshgen.forward_step(h=1.0 / 30)
    far = np.array(primitive_to_conservative(1.4, 3.0, 0.0, 1.0))
    U0 = np.zeros((4, 3, mesh.ntri))
    U0[:, 0, :] = far[:, None]
    path = str(tmp_path / "step.ckpt")
    a = CUDARkdgSolver(mesh, order=1, nq=3, ng=2, flux="llf", rk=3, limiter="tvb", tvb_m=50.0,
                       precision="fp32", cfl=0.3, farfield=far)
    a.setFreedom(U0, basis="native")
    a.advance(10 ** 6, t_final=0.004)
    a.checkpoint(path)
    a.advance(10 ** 6, t_final=0.01)
    ref = a.copyFreedomToHost(basis="native")
    b = CUDARkdgSolver(mesh, order=1, nq=3, ng=2, flux="llf", rk=3, limiter="tvb", tvb_m=50.0,
                       precision="fp32", cfl=0.3, farfield=far)
    b.restore(path)
    t, _ = b.advance(10 ** 6, t_final=0.01)
    assert t == 0.01
    np.testing.assert_array_equal(b.copyFreedomToHost(basis="native"), ref)


def test_mismatched_checkpoints_are_refused(tmp_path):
    mesh = meshgen.periodic_delaunay(12, seed=1)
    U0 = vortex.project_native(mesh, lambda X, Y: vortex.exact(X, Y, 0.0), 6)
    path = str(tmp_path / "a.ckpt")
    a = solver(mesh, "fp32")
    a.setFreedom(U0, basis="native")
    a.checkpoint(path)
    for other in (solver(meshgen.periodic_delaunay(12, seed=2), "fp32"),   # another mesh, same size
                  solver(mesh, "fp64"),                                      # another precision
                  solver(mesh, "fp32", order=1),                             # another order
                  solver(mesh, "fp32", far=primitive_to_conservative(1.0, 0.5, 0.0, 1.0)),
                  # another flux, CFL number or gamma: the saved wave maximum and state belong to
                  # the writer's method and physics
                  CUDARkdgSolver(mesh, order=2, nq=6, ng=3, flux="llf", rk=3, precision="fp32", cfl=0.2,
                                 farfield=FAR),
                  CUDARkdgSolver(mesh, order=2, nq=6, ng=3, flux="hllc", rk=3, precision="fp32", cfl=0.3,
                                 farfield=FAR),
                  CUDARkdgSolver(mesh, order=2, nq=6, ng=3, flux="hllc", rk=3, precision="fp32", cfl=0.2,
                                 farfield=FAR, gamma=1.3)):
        with pytest.raises(capi.RkdgError) as e:
            other.restore(path)
        assert e.value.code == capi.RKDG_ERR_INVALID
    with pytest.raises(capi.RkdgError) as e:
        a.restore(str(tmp_path / "missing.ckpt"))
    assert e.value.code == capi.RKDG_ERR_IO


def test_device_wait_gives_up_and_the_device_stays_usable():
    """A staging wait on data that never arrives ends after its limit with a
    status the host reads (no hang), and the next solve runs normally."""
    import ctypes as C

    t, w = C.c_int32(), C.c_double()
    capi.check(capi.lib().rkdg_wait_selftest(0.2, C.byref(t), C.byref(w)))
    assert t.value == 1 and 0.2 <= w.value < 5.0
    mesh = meshgen.periodic_delaunay(8, seed=1)
    s = solver(mesh, "fp32")
    s.initRKDG()
    s.advance(3)
    U = s.copyFreedomToHost(basis="native")
    assert np.abs(U[:, 0, :] - np.array(FAR)[:, None]).max() < 1e-6
