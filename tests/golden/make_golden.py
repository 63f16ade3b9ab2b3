"""Generates the golden fixtures of tests/golden/ by running the REFERENCE's
own RKDG code (multi_gpuRkdg sources compiled for the host into
oracle/_ref/librkdg_ref.so by oracle/Makefile) on small seeded meshes.

    make -C oracle libref && python tests/golden/make_golden.py

It also stores the reference's own NACA0012 mesh set (input/previous/ of the
checkout: vertices, triangles and neighbours as its files give them, and
the boundary tags of its |x|,|y| > 15 far-field rule) as
naca0012_previous.npz, the mesh the C++ caller test drives through the C
ABI where the checkout is absent.

Each vortex/box .npz holds the mesh (vertices, triangles, neighbours, boundary tags),
the reference-native parameters (P2, 7-point volume rule, 3-point edges,
LLF, SSP-RK3), an initial state in the reference basis, and the reference's
outputs: dt, R(U0), the state after each of the three stages of the first
step, the residual monitor of that step, and the state and dts after five
full steps.  The fixtures let the oracle be checked where the reference
cannot be built (no reference checkout).
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from helpers import perturbed_state, vortex_state  # noqa: E402
from oracle import oracle, ref  # noqa: E402
from rkdg_heter_calculate_b200 import meshgen  # noqa: E402
from rkdg_heter_calculate_b200.solver import freestream_state  # noqa: E402


def run_case(name, mesh, alpha_deg, mach, state_fn):
    gamma, cfl = 1.4, 0.18
    far = freestream_state(gamma, mach, alpha_deg)
    r = ref.RefCase(mesh, gamma=gamma, alpha_deg=alpha_deg, mach=mach, cfl=cfl)
    o = oracle.Oracle(mesh, farfield=far, cfl=cfl, gamma=gamma)
    coeff = o.basis()["coeff"]
    U0 = state_fn(mesh, coeff)
    r.set_dofs(U0)
    R0 = r.residual()
    dt0 = r.time_step()
    r.set_dofs(U0)
    r.save_old()
    stages = []
    for s in range(3):
        r.stage(s, dt0)
        stages.append(r.dofs())
    r.set_dofs(U0)
    dts1, res1 = r.advance(1)
    r.set_dofs(U0)
    dts5, res5 = r.advance(5)
    U5 = r.dofs()
    out = os.path.join(HERE, name + ".npz")
    np.savez_compressed(out, vertices=mesh.vertices, tris=mesh.tris, neighbours=mesh.neighbours,
                        bc=mesh.bc, periodic=mesh.periodic, gamma=gamma, cfl=cfl,
                        farfield=np.array(far), alpha_deg=alpha_deg, mach=mach, U0=U0, R0=R0,
                        dt0=dt0, stage1=stages[0], stage2=stages[1], stage3=stages[2],
                        monitor1=res1[0], dts5=dts5, U5=U5)
    print(out, mesh.ntri, "tris, dt0", dt0, "monitor", res1[0])


def naca_fixture():
    """The reference's NACA0012 mesh set, read by the library's reader of its
    file format (rkdg_read_mesh) from the checkout."""
    from rkdg_heter_calculate_b200 import capi

    src = os.path.join(ref.reference_dir(), "input", "previous")
    with tempfile.TemporaryDirectory() as d:
        os.symlink(src, os.path.join(d, "input"))
        V, T, N = capi.read_mesh(d, "input/mesh.conf")
    nb, _, bc = capi.build_connectivity(V, T)
    assert (nb == N).all()
    out = os.path.join(HERE, "naca0012_previous.npz")
    np.savez_compressed(out, vertices=V, tris=T.astype(np.int32), neighbours=N.astype(np.int32),
                        bc=bc.astype(np.int8))
    print(out, T.shape[0], "tris,", V.shape[0], "vertices")


def main():
    naca_fixture()
    m1 = meshgen.periodic_structured(8, 8, jitter=0.15, seed=5)
    run_case("periodic_8x8_vortex", m1, 45.0, 0.4,
             lambda m, c: vortex_state(m, c, 6))
    m2 = meshgen.box_with_obstacle(n=12, half=20.0, hole=1, jitter=0.2, seed=7)
    far = freestream_state(1.4, 0.4, 5.0)
    run_case("box_obstacle_12", m2, 5.0, 0.4, lambda m, c: perturbed_state(m, c, 6, far))


if __name__ == "__main__":
    main()
