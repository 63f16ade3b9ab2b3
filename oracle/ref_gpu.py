"""ctypes wrapper of the reference's OWN CUDA code built for the B200
(oracle/_ref/gpu/librkdg_ref_gpu.so, made by `make -C oracle libref_gpu`
from the reference checkout; see ref_gpu_harness.cu).

Test infrastructure: the check that the reference's kernels, run on the
device, agree with its host-compiled build, the residual comparison with
this library, the byte comparison of the solution writer, and the step-rate
comparison printed by tests/test_gpu_reference_kernels.py.  The product
library and the benchmark never call it.
"""
from __future__ import annotations

import ctypes as C
import os
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "gpu", "librkdg_ref_gpu.so")
_dp = C.POINTER(C.c_double)
_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"{LIB_PATH} not built (make -C oracle libref_gpu)")
        L = C.CDLL(LIB_PATH)
        L.rkdg_refgpu_open.restype = C.c_void_p
        L.rkdg_refgpu_open.argtypes = [C.c_char_p, C.c_char_p, _dp, C.c_int, C.c_char_p, C.c_int]
        L.rkdg_refgpu_close.argtypes = [C.c_void_p]
        L.rkdg_refgpu_sizes.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.rkdg_refgpu_set_dofs.argtypes = [C.c_void_p, _dp]
        L.rkdg_refgpu_get_dofs.argtypes = [C.c_void_p, _dp]
        L.rkdg_refgpu_residual.argtypes = [C.c_void_p, _dp]
        L.rkdg_refgpu_steps.argtypes = [C.c_void_p, C.c_int, _dp, _dp]
        L.rkdg_refgpu_write_solution.argtypes = [C.c_void_p, _dp, C.c_char_p]
        _lib = L
    return _lib


class RefGpuCase:
    """The reference's CCUDARkdgSolver on one mesh, on the current device."""

    def __init__(self, mesh, gamma=1.4, alpha_deg=0.0, mach=0.4, cfl=0.18, rhoref=1.0, pref=1.0,
                 threads_per_block=512):
        from rkdg_heter_calculate_b200 import meshgen

        self._tmp = tempfile.TemporaryDirectory(prefix="rkdg_refgpu_")
        conf = meshgen.write_reference_format(mesh, self._tmp.name)
        params = np.array([gamma, alpha_deg, mach, cfl, rhoref, pref], dtype=np.float64)
        err = C.create_string_buffer(512)
        h = lib().rkdg_refgpu_open(self._tmp.name.encode(), conf.encode(), params.ctypes.data_as(_dp),
                                   threads_per_block, err, 512)
        if not h:
            raise RuntimeError("reference GPU set-up failed: " + err.value.decode(errors="replace"))
        self.h = C.c_void_p(h)
        t, n = C.c_int(), C.c_int()
        lib().rkdg_refgpu_sizes(self.h, C.byref(t), C.byref(n))
        self.tnum, self.num = t.value, n.value

    def close(self):
        if getattr(self, "h", None):
            lib().rkdg_refgpu_close(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, U):
        """U: [4][6][tnum] in the reference basis (ghost cells are refilled by its boundary kernel)."""
        full = np.zeros((4, 6, self.num))
        full[:, :, : U.shape[2]] = U
        full = np.ascontiguousarray(full)
        assert lib().rkdg_refgpu_set_dofs(self.h, full.ctypes.data_as(_dp)) == 0

    def state(self):
        out = np.zeros((4, 6, self.num))
        assert lib().rkdg_refgpu_get_dofs(self.h, out.ctypes.data_as(_dp)) == 0
        return out[:, :, : self.tnum]

    def residual(self):
        out = np.zeros((4, 6, self.num))
        assert lib().rkdg_refgpu_residual(self.h, out.ctypes.data_as(_dp)) == 0
        return out[:, :, : self.tnum]

    def write_solution(self, means, path: str):
        """The reference's own solution.plt writer (CCUDARkdgSolver::
        outputSolution) on this mesh with the cell means [4][tnum]."""
        m = np.ascontiguousarray(means, dtype=np.float64)
        assert m.shape == (4, self.tnum)
        assert lib().rkdg_refgpu_write_solution(self.h, m.ctypes.data_as(_dp), path.encode()) == 0

    def steps(self, n: int):
        """n steps; returns (device ms, last dt)."""
        ms, dt = C.c_double(), C.c_double()
        assert lib().rkdg_refgpu_steps(self.h, int(n), C.byref(ms), C.byref(dt)) == 0
        return ms.value, dt.value
