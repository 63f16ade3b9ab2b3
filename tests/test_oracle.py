"""The oracle (plain-C restatement) pinned against the reference itself:
against the golden fixtures that the compiled reference produced
(tests/golden/make_golden.py), and, where the reference checkout and
oracle/_ref are present, against the compiled reference directly."""
import os

import numpy as np
import pytest

from helpers import perturbed_state, rel_err, vortex_state
from oracle import oracle, ref
from rkdg_heter_calculate_b200 import meshgen
from rkdg_heter_calculate_b200.solver import freestream_state

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
FIXTURES = ["periodic_8x8_vortex", "box_obstacle_12"]
TOL = 1e-12  # FP64 parity bar, relative to the largest |value| per variable


def load_fixture(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    mesh = meshgen.Mesh(z["vertices"], z["tris"], z["neighbours"], z["bc"], bool(z["periodic"]), name)
    return z, mesh


def make_oracle(z, mesh, **kw):
    return oracle.Oracle(mesh, order=2, nq=7, ng=3, flux=oracle.LLF, rk=3, gamma=float(z["gamma"]),
                         cfl=float(z["cfl"]), farfield=tuple(z["farfield"]), **kw)


@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_matches_golden_residual_and_dt(name):
    z, mesh = load_fixture(name)
    o = make_oracle(z, mesh)
    o.set_state(z["U0"])
    assert rel_err(o.residual(), z["R0"]) < TOL
    assert abs(o.time_step() - float(z["dt0"])) <= 1e-15 * float(z["dt0"])


@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_matches_golden_stages(name):
    z, mesh = load_fixture(name)
    o = make_oracle(z, mesh)
    o.set_state(z["U0"])
    o.save_old()
    dt = float(z["dt0"])
    for s, key in enumerate(["stage1", "stage2", "stage3"]):
        o.stage(s, dt)
        assert rel_err(o.state(), z[key]) < TOL, key


@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_matches_golden_steps(name):
    z, mesh = load_fixture(name)
    o = make_oracle(z, mesh)
    o.set_state(z["U0"])
    dt, mon = o.step()
    assert dt == pytest.approx(float(z["dt0"]), rel=1e-15)
    np.testing.assert_allclose(mon, z["monitor1"], rtol=1e-11)
    o.set_state(z["U0"])
    for k in range(5):
        dt, _ = o.step()
        assert dt == pytest.approx(float(z["dts5"][k]), rel=1e-12)
    assert rel_err(o.state(), z["U5"]) < 1e-11


needs_ref = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built (no reference checkout)")


@needs_ref
@pytest.mark.parametrize("seed", [1, 2])
def test_oracle_matches_compiled_reference(seed):
    mesh = meshgen.periodic_structured(10, 7, L=10.0, jitter=0.2, seed=seed)
    r = ref.RefCase(mesh, alpha_deg=30.0, mach=0.5)
    o = oracle.Oracle(mesh, farfield=freestream_state(1.4, 0.5, 30.0))
    g = r.geometry()
    b = o.basis()
    T = mesh.ntri
    np.testing.assert_allclose(b["area"], g["area"][:T], rtol=1e-15)
    np.testing.assert_allclose(b["mass"].T, g["mass"][:, :T], rtol=1e-12)
    U0 = vortex_state(mesh, b["coeff"], 6, beta=3.0)
    r.set_dofs(U0)
    o.set_state(U0)
    assert rel_err(o.residual(), r.residual()) < TOL
    dts, res = r.advance(4)
    for k in range(4):
        dt, mon = o.step()
        assert dt == pytest.approx(dts[k], rel=1e-13)
    assert rel_err(o.state(), r.dofs()) < TOL


@needs_ref
def test_oracle_matches_compiled_reference_walls_farfield():
    mesh = meshgen.box_with_obstacle(n=10, half=20.0, hole=1, jitter=0.25, seed=3)
    far = freestream_state(1.4, 0.6, -10.0)
    r = ref.RefCase(mesh, alpha_deg=-10.0, mach=0.6)
    o = oracle.Oracle(mesh, farfield=far)
    U0 = perturbed_state(mesh, o.basis()["coeff"], 6, far, amp=0.1)
    r.set_dofs(U0)
    o.set_state(U0)
    assert rel_err(o.residual(), r.residual()) < TOL
    r.advance(3)
    for _ in range(3):
        o.step()
    assert rel_err(o.state(), r.dofs()) < TOL
