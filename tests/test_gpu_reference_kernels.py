"""The reference's own CUDA kernels, built from its sources for the B200
(oracle/_ref/gpu, `make -C oracle libref_gpu`), against its host-compiled
build and against this library: R(U) to 1e-12, the first step's dt and
state, and the step rate of both on the same mesh and method (printed; this
library must be faster)."""
import time

import numpy as np
import pytest

from helpers import rel_err, vortex_state
from oracle import oracle, ref, ref_gpu
from rkdg_heter_calculate_b200 import CUDARkdgSolver, meshgen
from rkdg_heter_calculate_b200.solver import freestream_state

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (ref_gpu.available() and ref.available()),
                                 reason="the reference's GPU build (oracle/_ref/gpu) is absent")]


def test_reference_kernels_on_the_gpu_match_its_host_build():
    mesh = meshgen.box_with_obstacle(n=10, half=20.0, hole=1, jitter=0.25, seed=3)
    r = ref.RefCase(mesh, alpha_deg=-10.0, mach=0.6)
    g = ref_gpu.RefGpuCase(mesh, alpha_deg=-10.0, mach=0.6)
    o = oracle.Oracle(mesh, farfield=freestream_state(1.4, 0.6, -10.0))
    U0 = vortex_state(mesh, o.basis()["coeff"], 6, beta=2.0, uinf=0.5, vinf=-0.1)
    r.set_dofs(U0)
    g.set_state(U0)
    assert rel_err(g.residual(), r.residual()) < 1e-12
    g.set_state(U0)
    dts, _ = r.advance(1)
    _, dt = g.steps(1)
    assert dt == pytest.approx(dts[0], rel=1e-13)
    assert rel_err(g.state(), r.dofs()) < 1e-12


def test_step_rate_against_the_reference_kernels():
    mesh = meshgen.periodic_delaunay(120, L=10.0, jitter=0.3, seed=2)
    far = freestream_state(1.4, 0.4, 5.0)
    g = ref_gpu.RefGpuCase(mesh, alpha_deg=5.0, mach=0.4, cfl=0.18)
    g.steps(20)
    ms_ref, _ = g.steps(20)
    s = CUDARkdgSolver(mesh, order=2, nq=7, ng=3, flux="llf", rk=3, precision="fp64", cfl=0.18,
                       farfield=far)
    s.initRKDG()
    s.advance(20)  # warm: the step graphs are captured on the first advance long enough to use them
    import torch

    st = torch.cuda.ExternalStream(s.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    s.advance(20)
    e1.record(st)
    torch.cuda.synchronize()
    ms_ours = e0.elapsed_time(e1)
    unit = mesh.ntri * 24 * 3 * 20
    print(f"\n{mesh.ntri} triangles, P2 7/3-point LLF SSP-RK3 FP64: reference kernels "
          f"{unit / (ms_ref * 1e-3):.3e} DOF-stage/s ({ms_ref / 20:.3f} ms/step), this library "
          f"{unit / (ms_ours * 1e-3):.3e} DOF-stage/s ({ms_ours / 20:.3f} ms/step), "
          f"ratio {ms_ref / ms_ours:.1f}")
    assert ms_ours < ms_ref
    s.close()
    g.close()
