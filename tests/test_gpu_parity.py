"""Parity of the CUDA path (through the C ABI) with the reference and the
oracle, FP64 at 1e-12 relative per stage (normwise per variable: max |a-b|
over max |b|), FP32 at the tolerance stated per test."""
import os

import numpy as np
import pytest

from helpers import perturbed_state, rel_err, vortex_state
from oracle import oracle
from rkdg_heter_calculate_b200 import CUDARkdgSolver, meshgen
from rkdg_heter_calculate_b200.solver import freestream_state, primitive_to_conservative

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
FIXTURES = ["periodic_8x8_vortex", "box_obstacle_12"]
TOL64 = 1e-12


def load_fixture(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    mesh = meshgen.Mesh(z["vertices"], z["tris"], z["neighbours"], z["bc"], bool(z["periodic"]), name)
    return z, mesh


def gpu_from_fixture(z, mesh, precision="fp64", reorder=True):
    return CUDARkdgSolver(mesh, order=2, nq=7, ng=3, flux="llf", rk=3, precision=precision,
                          gamma=float(z["gamma"]), cfl=float(z["cfl"]),
                          farfield=tuple(z["farfield"]), reorder=reorder)


# ------------------------------------------------- against the reference --
@pytest.mark.parametrize("name", FIXTURES)
@pytest.mark.parametrize("reorder", [True, False])
def test_residual_matches_reference(name, reorder):
    z, mesh = load_fixture(name)
    s = gpu_from_fixture(z, mesh, reorder=reorder)
    s.setFreedom(z["U0"])
    np.testing.assert_allclose(s.copyFreedomToHost(), z["U0"], rtol=0,
                               atol=1e-13 * np.abs(z["U0"]).max())
    assert rel_err(s.residual(), z["R0"]) < TOL64
    assert s.getTimeStep() == pytest.approx(float(z["dt0"]), rel=1e-13)


@pytest.mark.parametrize("name", FIXTURES)
def test_stages_match_reference(name):
    z, mesh = load_fixture(name)
    s = gpu_from_fixture(z, mesh)
    s.setFreedom(z["U0"])
    s.saveOld()
    dt = float(z["dt0"])
    for k, key in enumerate(["stage1", "stage2", "stage3"]):
        s.stage(k, dt)
        assert rel_err(s.copyFreedomToHost(), z[key]) < TOL64, key


@pytest.mark.parametrize("name", FIXTURES)
def test_steps_match_reference(name):
    z, mesh = load_fixture(name)
    s = gpu_from_fixture(z, mesh)
    s.setFreedom(z["U0"])
    dt, mon = s.step()
    assert dt == pytest.approx(float(z["dt0"]), rel=1e-13)
    np.testing.assert_allclose(mon, z["monitor1"], rtol=1e-10)
    s.setFreedom(z["U0"])
    s.set_time(0.0)
    t, n = s.advance(5)
    assert n == 5
    assert t == pytest.approx(float(z["dts5"].sum()), rel=1e-12)
    assert rel_err(s.copyFreedomToHost(), z["U5"]) < 1e-11


# ----------------------------------------------------- against the oracle --
CONFIGS = [
    ("p2_llf_rk3_ref", dict(order=2, nq=7, ng=3, flux="llf", rk=3)),
    ("p2_hllc_rk3", dict(order=2, nq=6, ng=3, flux="hllc", rk=3)),
    ("p1_llf_rk2", dict(order=1, nq=3, ng=2, flux="llf", rk=2)),
    ("p1_hllc_rk3", dict(order=1, nq=3, ng=2, flux="hllc", rk=3)),
]


def oracle_for(mesh, cfg, far, **kw):
    return oracle.Oracle(mesh, order=cfg["order"], nq=cfg["nq"], ng=cfg["ng"],
                         flux=oracle.HLLC if cfg["flux"] == "hllc" else oracle.LLF, rk=cfg["rk"],
                         farfield=far, **kw)


@pytest.mark.parametrize("label,cfg", CONFIGS)
def test_vortex_matches_oracle(label, cfg):
    mesh = meshgen.periodic_delaunay(14, seed=2)
    far = primitive_to_conservative(1.0, 1.0, 1.0, 1.0)
    o = oracle_for(mesh, cfg, far, cfl=0.3)
    nb = o.nb
    U0 = vortex_state(mesh, o.basis()["coeff"], nb)
    s = CUDARkdgSolver(mesh, cfl=0.3, farfield=far, **cfg)
    s.setFreedom(U0)
    o.set_state(U0)
    assert rel_err(s.residual(), o.residual()) < TOL64
    for _ in range(10):
        dt_o, mon_o = o.step()
        dt_g, mon_g = s.step()
        assert dt_g == pytest.approx(dt_o, rel=1e-12)
    assert rel_err(s.copyFreedomToHost(), o.state()) < 1e-11


def test_plain_p1_rk2_vortex_100_steps():
    """The plain-method configuration: 40 x 40 periodic squares split into 3,200
    triangles, P1, 3-point volume / 2-point edge rules, LLF, SSP-RK2, CFL 0.3,
    100 steps of the strength-5 vortex; every step's dt and the final state
    against the oracle, and the vortex L2(rho) error of both against the exact
    solution."""
    from rkdg_heter_calculate_b200 import vortex

    mesh = meshgen.periodic_structured(40, 40)
    assert mesh.ntri == 3200
    far = primitive_to_conservative(1.0, 1.0, 1.0, 1.0)
    cfg = dict(order=1, nq=3, ng=2, flux="llf", rk=2)
    o = oracle_for(mesh, cfg, far, cfl=0.3)
    U0 = vortex_state(mesh, o.basis()["coeff"], 3)
    s = CUDARkdgSolver(mesh, cfl=0.3, farfield=far, **cfg)
    s.setFreedom(U0)
    o.set_state(U0)
    t = 0.0
    for _ in range(100):
        dt_o, _ = o.step()
        dt_g, _ = s.step()
        assert dt_g == pytest.approx(dt_o, rel=1e-12)
        t += dt_o
    assert rel_err(s.copyFreedomToHost(), o.state()) < 1e-11
    native = s.copyFreedomToHost(basis="native")
    err = vortex.l2_error(mesh, native, lambda X, Y: vortex.exact(X, Y, t))
    assert 0.0 < err < 0.1  # P1 on h = 0.25: resolved, visibly diffused


@pytest.mark.parametrize("label,cfg", CONFIGS)
def test_boundaries_match_oracle(label, cfg):
    mesh = meshgen.channel(18, 6, jitter=0.25, seed=5)
    far = primitive_to_conservative(1.0, 0.8, 0.1, 1.0)
    o = oracle_for(mesh, cfg, far, cfl=0.2)
    U0 = perturbed_state(mesh, o.basis()["coeff"], o.nb, far, amp=0.1)
    s = CUDARkdgSolver(mesh, cfl=0.2, farfield=far, **cfg)
    s.setFreedom(U0)
    o.set_state(U0)
    assert rel_err(s.residual(), o.residual()) < TOL64
    for _ in range(8):
        o.step()
        s.step()
    assert rel_err(s.copyFreedomToHost(), o.state()) < 1e-11


def test_limiter_matches_oracle():
    mesh = meshgen.channel(40, 14, jitter=0.2, seed=8)
    far = primitive_to_conservative(1.4, 3.0, 0.0, 1.0)
    o = oracle.Oracle(mesh, order=1, nq=3, ng=2, flux=oracle.LLF, rk=3,
                      limiter=oracle.LIMITER_TVB, tvb_m=50.0, farfield=far, cfl=0.3)
    coeff = o.basis()["coeff"]

    def shock(X, Y):
        left = X + 0.2 * Y < 1.2
        r = np.where(left, 1.4, 3.0)
        u = np.where(left, 3.0, 1.2)
        p = np.where(left, 1.0, 4.0)
        return np.stack(primitive_to_conservative(r, u, 0 * X, p))

    from helpers import project_reference

    U0 = project_reference(mesh, shock, coeff, 3)
    s = CUDARkdgSolver(mesh, order=1, nq=3, ng=2, flux="llf", rk=3, limiter="tvb", tvb_m=50.0,
                       farfield=far, cfl=0.3)
    s.setFreedom(U0)
    o.set_state(U0)
    o.limit()
    s.limit()
    assert rel_err(s.copyFreedomToHost(), o.state()) < TOL64
    for _ in range(10):
        o.step()
        s.step()
    assert rel_err(s.copyFreedomToHost(), o.state()) < 1e-10


# -------------------------------------------------------- FP32 precision --
def test_fp32_tracks_fp64():
    """FP32 state and arithmetic (FP64 geometry and dt): 20 steps of the
    vortex agree with FP64 to 1e-5 relative."""
    mesh = meshgen.periodic_delaunay(14, seed=2)
    far = primitive_to_conservative(1.0, 1.0, 1.0, 1.0)
    o = oracle.Oracle(mesh, order=2, nq=6, ng=3, flux=oracle.HLLC, rk=3, farfield=far, cfl=0.2)
    U0 = vortex_state(mesh, o.basis()["coeff"], 6)
    a = CUDARkdgSolver(mesh, order=2, nq=6, ng=3, flux="hllc", precision="fp64", farfield=far, cfl=0.2)
    b = CUDARkdgSolver(mesh, order=2, nq=6, ng=3, flux="hllc", precision="fp32", farfield=far, cfl=0.2)
    a.setFreedom(U0)
    b.setFreedom(U0)
    assert rel_err(b.residual(), a.residual()) < 1e-5
    a.advance(20)
    b.advance(20)
    assert rel_err(b.copyFreedomToHost(), a.copyFreedomToHost()) < 1e-5


def test_fp32c_tracks_fp64_and_stops_the_storage_drift():
    """RKDG_FP32C (FP32 arithmetic; each cell mean a high + low float pair
    updated in FP64): it agrees with FP64 to 1e-5 like the FP32 form, and over
    300 steps of the vortex its cell means stay closer to the FP64 run's than
    the plain FP32 form's, whose mean storage rounding accumulates."""
    mesh = meshgen.periodic_delaunay(40, seed=2)
    far = primitive_to_conservative(1.0, 1.0, 1.0, 1.0)
    from rkdg_heter_calculate_b200 import vortex

    U0 = vortex.project_native(mesh, lambda X, Y: vortex.exact(X, Y, 0.0), 6, n=4)
    runs = {}
    for prec in ("fp64", "fp32", "fp32c"):
        s = CUDARkdgSolver(mesh, order=2, nq=6, ng=3, flux="hllc", precision=prec, farfield=far, cfl=0.2)
        s.setFreedom(U0, basis="native")
        s.advance(20)
        u20 = s.copyFreedomToHost(basis="native")
        s.advance(280)
        runs[prec] = (u20, s.copyFreedomToHost(basis="native"), s.time())
        s.close()
    assert rel_err(runs["fp32c"][0], runs["fp64"][0]) < 1e-5
    assert runs["fp32c"][2][1] == runs["fp64"][2][1] == 300
    d32 = np.abs(runs["fp32"][1][:, 0] - runs["fp64"][1][:, 0]).max()
    d32c = np.abs(runs["fp32c"][1][:, 0] - runs["fp64"][1][:, 0]).max()
    print(f"max |mean - FP64 mean| after 300 steps: FP32 {d32:.3e}, FP32C {d32c:.3e}")
    assert d32c < 0.5 * d32


# ------------------------------------------------------- properties -------
def test_free_stream_preserved_and_conservation():
    mesh = meshgen.periodic_delaunay(16, seed=4)
    far = primitive_to_conservative(1.1, 0.6, -0.3, 0.8)
    s = CUDARkdgSolver(mesh, order=2, nq=6, ng=3, flux="hllc", farfield=far)
    s.initRKDG()
    s.advance(5)
    U = s.copyFreedomToHost(basis="native")
    assert np.abs(U[:, 0, :] - np.array(far)[:, None]).max() < 1e-13
    assert np.abs(U[:, 1:, :]).max() < 1e-13
    o = oracle.Oracle(mesh, order=2, nq=6, ng=3, flux=oracle.HLLC)
    s.setFreedom(vortex_state(mesh, o.basis()["coeff"], 6))
    tot0 = s.conservation_totals()
    s.advance(10)
    np.testing.assert_allclose(s.conservation_totals(), tot0, rtol=1e-13)


@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp32c"])
def test_full_size_free_stream_and_conservation(precision):
    """At the unstructured-vortex size (700 x 700 lattice, 980,000 triangles,
    P2, HLLC): a uniform state stays uniform and the vortex's conserved totals
    stay constant over 20 steps (periodic mesh, FP64 totals of the FP64 or
    FP32 state)."""
    from rkdg_heter_calculate_b200 import vortex

    mesh = meshgen.periodic_delaunay(700, L=10.0, jitter=0.3, seed=2)
    assert mesh.ntri == 980000
    far = primitive_to_conservative(1.0, 1.0, 1.0, 1.0)
    s = CUDARkdgSolver(mesh, order=2, nq=6, ng=3, flux="hllc", precision=precision, cfl=0.2,
                       farfield=far)
    s.initRKDG()
    s.advance(20)
    U = s.copyFreedomToHost(basis="native")
    tol = 1e-13 if precision == "fp64" else 1e-6
    assert np.abs(U[:, 0, :] - np.array(far)[:, None]).max() < tol
    assert np.abs(U[:, 1:, :]).max() < tol
    s.setFreedom(vortex.project_native(mesh, lambda X, Y: vortex.exact(X, Y, 0.0), 6, n=2), basis="native")
    tot0 = s.conservation_totals()
    s.advance(20)
    np.testing.assert_allclose(s.conservation_totals(), tot0, rtol=1e-12 if precision == "fp64" else 1e-6)


def test_advance_lands_on_final_time():
    mesh = meshgen.periodic_structured(10, 10)
    s = CUDARkdgSolver(mesh, order=1, nq=3, ng=2, rk=2, cfl=0.3,
                       farfield=primitive_to_conservative(1.0, 1.0, 1.0, 1.0))
    o = oracle.Oracle(mesh, order=1, nq=3, ng=2, rk=2)
    s.setFreedom(vortex_state(mesh, o.basis()["coeff"], 3))
    t, n = s.advance(100000, t_final=0.1)
    assert t == 0.1 and n > 1
    t2, n2 = s.advance(10, t_final=0.1)
    assert t2 == 0.1 and n2 == 0


def test_nonphysical_state_is_reported():
    from rkdg_heter_calculate_b200 import RkdgError

    mesh = meshgen.periodic_structured(4, 4)
    s = CUDARkdgSolver(mesh, order=1, nq=3, ng=2)
    U = np.zeros((4, 3, mesh.ntri))
    U[0, 0] = 1.0
    U[3, 0] = 2.5
    U[0, 0, 3] = -1.0  # negative density in one cell
    s.setFreedom(U, basis="native")
    with pytest.raises(RkdgError) as e:
        s.getTimeStep()
    assert e.value.code == 4
    with pytest.raises(RkdgError):
        s.advance(3)


def test_residual_history_file(tmp_path):
    """The reference's residual history: header "N, rho", then one line per
    step with log10 of the largest cell-mean density change over the step
    (relative to the far-field density), through rkdg_step and rkdg_advance."""
    import math

    mesh = meshgen.periodic_delaunay(10, seed=3)
    far = primitive_to_conservative(1.2, 1.0, 1.0, 1.0)
    o = oracle.Oracle(mesh, order=2, nq=6, ng=3, flux=oracle.HLLC, rk=3, farfield=far, cfl=0.2)
    s = CUDARkdgSolver(mesh, order=2, nq=6, ng=3, flux="hllc", farfield=far, cfl=0.2)
    s.setFreedom(vortex_state(mesh, o.basis()["coeff"], 6))
    path = tmp_path / "residual.dat"
    s.setResidualLog(str(path))
    mons = [s.step()[1][0] for _ in range(2)]
    t, n = s.advance(5)
    s.setResidualLog(None)
    s.step()  # not logged
    lines = path.read_text().splitlines()
    assert lines[0] == "N, rho"
    assert len(lines) == 1 + 2 + 5
    steps = [int(x.split()[0]) for x in lines[1:]]
    assert steps == list(range(1, 8))
    for line, m in zip(lines[1:3], mons):
        assert float(line.split()[1]) == pytest.approx(math.log10(m / far[0]), rel=1e-9)
    assert all(math.isfinite(float(x.split()[1])) for x in lines[1:])


def test_solution_file_format(tmp_path):
    z, mesh = load_fixture("box_obstacle_12")
    s = gpu_from_fixture(z, mesh)
    s.setFreedom(z["U0"])
    path = str(tmp_path / "solution.plt")
    s.outputSolution(path)
    lines = open(path).read().split("\n")
    assert lines[0] == "TITLE=RKDG"
    assert lines[1] == "VARIABLES=X , Y , rho , u , v , p, Ma , FLAG"
    V, T = mesh.vertices.shape[0], mesh.ntri
    assert lines[2] == f"ZONE T= T1 N= {V} , E= {T} , ZONETYPE=FETRIANGLE"
    conn = [l for l in lines if l.count("    ") == 2]
    assert len(conn) == T
    assert [int(x) for x in conn[0].split()] == list(mesh.tris[0] + 1)
