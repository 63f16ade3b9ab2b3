"""The drop-in boundary driven from C++ and the reference's output format.

A C++ program (tests/cpp/reference_sequence.cpp) that keeps the reference's
call sequence (multi_gpuRkdg/src/main.cpp:56-149) is compiled with g++
against include/rkdg.h and librkdg.so and run on the reference's own
NACA0012 mesh set (fixture tests/golden/naca0012_previous.npz, written back
in the reference's file format): its final state equals the same sequence
through the Python binding bit for bit, and matches the oracle and the
reference's own code built for the host (oracle/_ref) after twenty steps to
1e-11; the reference's CUDA kernels (oracle/_ref/gpu) give the same
residual on it.  Its solution.plt
is byte-identical to the file the reference's own writer
(CCUDARkdgSolver::outputSolution, src/cudarkdgsolver.cu:860-1001) makes
from the same cell means.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

from helpers import rel_err
from oracle import oracle, ref, ref_gpu
from rkdg_heter_calculate_b200 import CUDARkdgSolver, meshgen
from rkdg_heter_calculate_b200.solver import freestream_state

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "rkdg_heter_calculate_b200")
NSTEPS = 20


def naca_mesh():
    z = np.load(os.path.join(ROOT, "tests", "golden", "naca0012_previous.npz"))
    m = meshgen.Mesh(vertices=z["vertices"], tris=z["tris"], neighbours=z["neighbours"], bc=z["bc"],
                     periodic=False, name="naca0012")
    m.check()
    return m


@pytest.fixture(scope="module")
def cpp_run(tmp_path_factory):
    """Compiles the C++ caller and runs it in a directory holding the NACA
    mesh files; returns (workdir, mesh)."""
    if shutil.which("g++") is None:
        pytest.skip("g++ absent")
    work = tmp_path_factory.mktemp("cpp_caller")
    mesh = naca_mesh()
    conf = meshgen.write_reference_format(mesh, str(work))
    assert conf == "input/mesh.conf"
    os.makedirs(work / "output")
    exe = str(work / "reference_sequence")
    subprocess.run(["g++", "-std=c++17", "-O2", os.path.join(ROOT, "tests", "cpp", "reference_sequence.cpp"),
                    "-I", os.path.join(ROOT, "include"), "-L", PKG, "-lrkdg", f"-Wl,-rpath,{PKG}", "-o", exe],
                   check=True, capture_output=True, text=True)
    r = subprocess.run([exe, str(NSTEPS)], cwd=str(work), capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    return work, mesh


def read_state(work, name, T):
    return np.fromfile(str(work / "output" / name), dtype=np.float64).reshape(4, 6, T)


def test_cpp_caller_equals_python_binding(cpp_run):
    work, mesh = cpp_run
    T = mesh.ntri
    ntri, nb, steps, t, *tot = open(work / "output" / "summary.txt").read().split()
    assert (int(ntri), int(nb), int(steps)) == (T, 6, NSTEPS)
    s = CUDARkdgSolver(mesh)  # the reference's defaults, as rkdg_default_params
    s.initRKDG()
    t_py, n_py = s.advance(NSTEPS)
    assert n_py == NSTEPS and t_py == float(t)
    np.testing.assert_array_equal(s.copyFreedomToHost(), read_state(work, "state_reference.bin", T))
    np.testing.assert_array_equal(s.copyFreedomToHost(basis="native"), read_state(work, "state_native.bin", T))
    np.testing.assert_array_equal(s.conservation_totals(), np.array([float(x) for x in tot]))
    s.close()
    # the residual history: header and one line per step
    lines = open(work / "output" / "residual.dat").read().splitlines()
    assert lines[0] == "N, rho" and len(lines) == NSTEPS + 1


def test_cpp_caller_matches_oracle(cpp_run):
    work, mesh = cpp_run
    T = mesh.ntri
    far = freestream_state(1.4, 0.4, 5.0)
    o = oracle.Oracle(mesh, farfield=far, cfl=0.18)
    U0 = np.zeros((4, 6, T))
    U0[:, 0, :] = np.array(far)[:, None]
    o.set_state(U0)
    for _ in range(NSTEPS):
        o.step()
    U = read_state(work, "state_reference.bin", T)
    # twenty steps: rounding accumulates over the stages (the host build of
    # the reference and the oracle differ by 1e-12 here)
    assert rel_err(U, o.state()) < 1e-11
    assert np.abs(U[:, 1:]).max() > 1e-6  # the airfoil has disturbed the free stream


@pytest.mark.skipif(not ref.available(), reason="the reference's host build (oracle/_ref) is absent")
def test_cpp_caller_matches_reference_host_build(cpp_run):
    """The reference's own code compiled for the host (oracle/_ref), run the
    same twenty steps from the same free stream on the same mesh files."""
    work, mesh = cpp_run
    T = mesh.ntri
    far = freestream_state(1.4, 0.4, 5.0)
    r = ref.RefCase(mesh, alpha_deg=5.0, mach=0.4, cfl=0.18)
    U0 = np.zeros((4, 6, T))
    U0[:, 0, :] = np.array(far)[:, None]
    r.set_dofs(U0)
    r.advance(NSTEPS)
    assert rel_err(read_state(work, "state_reference.bin", T), r.dofs()) < 1e-11
    r.close()


@pytest.mark.skipif(not ref_gpu.available(), reason="the reference's GPU build (oracle/_ref/gpu) is absent")
def test_cpp_caller_matches_reference_kernels_and_writer(cpp_run):
    work, mesh = cpp_run
    T = mesh.ntri
    g = ref_gpu.RefGpuCase(mesh, alpha_deg=5.0, mach=0.4, cfl=0.18)
    # the reference's own kernels on the C++ caller's final state: the same
    # residual (its multi-step runs are not compared: its block reductions of
    # dt rely on implicit warp synchrony, which sm_100 does not give)
    U = read_state(work, "state_reference.bin", T)
    g.set_state(U)
    s = CUDARkdgSolver(mesh)
    s.setFreedom(U)
    assert rel_err(s.residual(), g.residual()) < 1e-10
    s.close()
    # the reference's writer on the C++ caller's cell means: the same bytes
    ref_plt = str(work / "output" / "solution_reference_writer.plt")
    g.write_solution(read_state(work, "state_native.bin", T)[:, 0, :], ref_plt)
    g.close()
    ours = open(work / "output" / "solution.plt", "rb").read()
    theirs = open(ref_plt, "rb").read()
    assert len(ours) > 100000
    assert ours == theirs
