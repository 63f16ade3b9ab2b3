"""Host-side logic of librkdg.so that needs no GPU: symbol table, error
paths, native basis, connectivity, locality order, mesh file reader."""
import os
import re
import tempfile

import numpy as np
import pytest

from oracle import ref
from rkdg_heter_calculate_b200 import capi, meshgen, vortex

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# the reference's NACA0012 mesh set (present where the reference checkout is)
REF_MESH = os.path.join(ref.reference_dir(), "input", "previous")


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if f.endswith(".h"):
            txt = open(os.path.join(inc, f)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names |= set(re.findall(r"\b(rkdg_\w+)\s*\(", txt))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    L = capi.lib()
    names = declared_symbols()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def gpu_present():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(gpu_present(), reason="checks the no-device error path")
def test_create_without_device_fails_loudly():
    from rkdg_heter_calculate_b200 import CUDARkdgSolver

    with pytest.raises(capi.RkdgError) as e:
        CUDARkdgSolver(meshgen.periodic_structured(3, 3))
    assert e.value.code == 5


def test_native_basis_is_orthonormal_and_hierarchical():
    xi, eta, w = vortex.triangle_rule(6)
    psi = capi.native_basis(6, xi, eta)
    G = np.einsum("q,qi,qj->ij", w, psi, psi)
    np.testing.assert_allclose(G, np.eye(6), atol=1e-14)
    np.testing.assert_allclose(psi[:, 0], 1.0, atol=1e-15)
    # P1 functions are linear: second differences along xi vanish
    a = capi.native_basis(3, np.array([0.1, 0.2, 0.3]), np.array([0.2, 0.2, 0.2]))
    np.testing.assert_allclose(a[0] - 2 * a[1] + a[2], 0.0, atol=1e-14)


def test_native_basis_structure_the_stage_kernel_relies_on():
    # the tile kernel forms the psi_0 term once per state and skips the
    # eta-derivative of psi_1; the library checks both on its tables, here
    # they are checked bit for bit on the basis values
    rng = np.random.default_rng(7)
    xi = rng.uniform(0, 1, 64)
    eta = rng.uniform(0, 1, 64) * (1 - xi)
    psi = capi.native_basis(6, xi, eta)
    assert (psi[:, 0] == psi[0, 0]).all()
    psi_shift = capi.native_basis(6, xi, rng.uniform(0, 1, 64) * (1 - xi))
    np.testing.assert_array_equal(psi[:, 1], psi_shift[:, 1])
    assert not np.array_equal(psi[:, 2], psi_shift[:, 2])


def test_connectivity_matches_generator():
    for m in (meshgen.box_with_obstacle(n=10), meshgen.channel(10, 4)):
        nb, sh, bc = capi.build_connectivity(m.vertices, m.tris, None, m.bc)
        np.testing.assert_array_equal(nb, m.neighbours)
        np.testing.assert_array_equal(sh, meshgen.shared_edges(m))
        np.testing.assert_array_equal(bc, m.bc)


def test_periodic_connectivity_is_taken_from_neighbours():
    m = meshgen.periodic_structured(5, 4, jitter=0.1)
    nb, sh, bc = capi.build_connectivity(m.vertices, m.tris, m.neighbours)
    np.testing.assert_array_equal(nb, m.neighbours)
    assert (sh >= 0).all() and (bc == 0).all()
    np.testing.assert_array_equal(sh, meshgen.shared_edges(m))


def test_reference_boundary_rule():
    # without tags the library applies the reference's ghost-barycentre rule:
    # far field outside |x|,|y| <= 15, wall inside
    m = meshgen.box_with_obstacle(n=12, half=20.0)
    _, _, bc = capi.build_connectivity(m.vertices, m.tris)
    np.testing.assert_array_equal(bc, m.bc)


def test_invalid_meshes_are_rejected():
    m = meshgen.channel(4, 2)
    bad = m.tris.copy()
    bad[0, [1, 2]] = bad[0, [2, 1]]  # clockwise
    with pytest.raises(capi.RkdgError) as e:
        capi.build_connectivity(m.vertices, bad)
    assert e.value.code == 1
    nb = m.neighbours.copy()
    nb[0, 0] = m.ntri + 5
    with pytest.raises(capi.RkdgError):
        capi.build_connectivity(m.vertices, m.tris, nb)
    with pytest.raises(capi.RkdgError):  # boundary edge without a tag
        capi.build_connectivity(m.vertices, m.tris, None, np.zeros_like(m.bc))


def test_locality_order_is_a_permutation_and_local():
    m = meshgen.periodic_delaunay(40, seed=2)
    perm = capi.locality_order(m.vertices, m.tris, m.neighbours)
    assert np.array_equal(np.sort(perm), np.arange(m.ntri))
    mm = meshgen.permute(m, perm)
    d_sorted = np.median(np.abs(mm.neighbours - np.arange(m.ntri)[:, None]))
    rng = np.random.default_rng(0)
    mr = meshgen.permute(m, rng.permutation(m.ntri))
    d_rand = np.median(np.abs(mr.neighbours - np.arange(m.ntri)[:, None]))
    assert d_sorted < 0.05 * d_rand


def test_reader_roundtrip_reference_format():
    m = meshgen.box_with_obstacle(n=8)
    with tempfile.TemporaryDirectory() as d:
        conf = meshgen.write_reference_format(m, d)
        V, T, N = capi.read_mesh(d, conf)
    np.testing.assert_allclose(V, m.vertices, rtol=0, atol=1e-15)
    np.testing.assert_array_equal(T, m.tris)
    np.testing.assert_array_equal(N, m.neighbours)


@pytest.mark.skipif(not os.path.isdir(REF_MESH), reason="reference checkout absent")
def test_reader_on_reference_naca_mesh():
    # the NACA0012 set's mesh.conf names input/*.dat relative to the run directory
    with tempfile.TemporaryDirectory() as d:
        os.symlink(REF_MESH, os.path.join(d, "input"))
        V, T, N = capi.read_mesh(d, "input/mesh.conf")
    assert V.shape == (4767, 2) and T.shape == (9340, 3)
    nb, sh, bc = capi.build_connectivity(V, T)  # rebuilt from vertex ids
    np.testing.assert_array_equal(nb, N)
    assert (bc[nb < 0] > 0).all() and (nb < 0).sum() == 194


def test_delaunay_generators():
    m = meshgen.periodic_delaunay(30, seed=2)
    assert m.ntri == 2 * 30 * 30 and (m.neighbours >= 0).all()
    s = meshgen.forward_step(h=1.0 / 40, seed=3)
    assert (s.bc[s.neighbours < 0] > 0).all()
    assert np.isclose(s.areas().sum(), 3.0 - 2.4 * 0.2)


def test_cpp_caller_compiles_and_links():
    """The C++ program that keeps the reference's call sequence
    (tests/cpp/reference_sequence.cpp) compiles against include/rkdg.h and
    links against librkdg.so; without its mesh files it reports the reader's
    error and exits non-zero (no device is touched)."""
    import shutil
    import subprocess

    if shutil.which("g++") is None:
        pytest.skip("g++ absent")
    pkg = os.path.join(ROOT, "rkdg_heter_calculate_b200")
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "reference_sequence")
        subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror",
                        os.path.join(ROOT, "tests", "cpp", "reference_sequence.cpp"),
                        "-I", os.path.join(ROOT, "include"), "-L", pkg, "-lrkdg", f"-Wl,-rpath,{pkg}",
                        "-o", exe], check=True, capture_output=True, text=True)
        r = subprocess.run([exe, "1"], cwd=d, capture_output=True, text=True, timeout=60)
        assert r.returncode == 1 and "rkdg_read_mesh" in r.stderr
