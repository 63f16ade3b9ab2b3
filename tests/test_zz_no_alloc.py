"""The allocation-free totals entry point against the context-based one.

rkdg_conservation_totals_noalloc exists for callers that cannot allocate
device memory (their device memory is owned by another allocator, or they
must not allocate once running): they hand in device inputs and an output
and the library uses a static device array as its scratch.  This file is
collected last so that a failure here comes after every other test has run;
it passes alone in a fresh process and after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from rkdg_heter_calculate_b200 import CUDARkdgSolver, capi, meshgen, vortex

pytestmark = pytest.mark.gpu


def _call(T, d_means, ld, d_area, d_out, stream):
    return capi.lib().rkdg_conservation_totals_noalloc(T, C.c_void_p(d_means), ld, C.c_void_p(d_area),
                                                       C.c_void_p(d_out), C.c_void_p(stream))


def test_noalloc_totals_match_context_totals_on_two_calls():
    import torch

    mesh = meshgen.periodic_delaunay(60, seed=3)
    T = mesh.ntri
    s = CUDARkdgSolver(mesh, order=2, nq=6, ng=3, flux="hllc", rk=3,
                       farfield=(1.0, 1.0, 1.0, 3.5))
    stream = torch.cuda.current_stream().cuda_stream
    for call, beta in enumerate((5.0, 2.0)):  # two calls in a row, different data
        U = vortex.project_native(mesh, lambda X, Y: vortex.exact(X, Y, 0.0, beta=beta), 6)
        s.setFreedom(U, basis="native")
        s.advance(3)
        expected = s.conservation_totals()  # existing entry point (context scratch)
        means = s.copyFreedomToHost(basis="native")[:, 0, :]  # cell means (4, T)
        ld = T + 7  # a padded leading dimension
        host = np.zeros((4, ld))
        host[:, :T] = means
        d_means = torch.tensor(host, dtype=torch.float64, device="cuda")
        d_area = torch.tensor(mesh.areas(), dtype=torch.float64, device="cuda")
        d_out = torch.full((4,), float("nan"), dtype=torch.float64, device="cuda")
        rc = _call(T, d_means.data_ptr(), ld, d_area.data_ptr(), d_out.data_ptr(), stream)
        assert rc == 0, capi.lib().rkdg_last_error()
        torch.cuda.synchronize()
        got = d_out.cpu().numpy()
        np.testing.assert_allclose(got, expected, rtol=1e-12, atol=0.0, err_msg=f"call {call}")
    s.close()


def test_noalloc_totals_in_place_on_a_full_state_and_its_own_stream():
    """A caller that keeps its whole state on the device in the reference
    layout [4][nbasis][ld] passes it in place: the mean rows (row 0 of each
    variable's block) are nbasis * ld apart, so d_means is the array itself
    with that stride.  The call is ordered on a stream the caller created."""
    import torch

    mesh = meshgen.periodic_delaunay(40, seed=8)
    T = mesh.ntri
    s = CUDARkdgSolver(mesh, order=2, nq=6, ng=3, flux="hllc", rk=3, farfield=(1.0, 1.0, 1.0, 3.5))
    U = vortex.project_native(mesh, lambda X, Y: vortex.exact(X, Y, 0.0, beta=4.0), 6)
    s.setFreedom(U, basis="native")
    s.advance(2)
    expected = s.conservation_totals()
    state = s.copyFreedomToHost(basis="native")  # [4][6][T]
    s.close()
    ld = T + 3
    full = np.zeros((4, 6, ld))
    full[:, :, :T] = state
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        d_state = torch.tensor(full, dtype=torch.float64, device="cuda")
        d_area = torch.tensor(mesh.areas(), dtype=torch.float64, device="cuda")
        d_out = torch.full((4,), float("nan"), dtype=torch.float64, device="cuda")
    rc = _call(T, d_state.data_ptr(), 6 * ld, d_area.data_ptr(), d_out.data_ptr(), stream.cuda_stream)
    assert rc == 0, capi.lib().rkdg_last_error()
    stream.synchronize()
    np.testing.assert_allclose(d_out.cpu().numpy(), expected, rtol=1e-12, atol=0.0)


def test_noalloc_rejects_oversized_meshes():
    rc = _call(4096 * 256 + 1, 1, 4096 * 256 + 1, 1, 1, 0)
    assert rc == capi.RKDG_OK + 1  # RKDG_ERR_INVALID, no launch
    assert b"exceeds the maximum" in capi.lib().rkdg_last_error()
