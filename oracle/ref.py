"""ctypes front-end of oracle/_ref/librkdg_ref.so -- the reference's own RKDG
code (multi_gpuRkdg/src/*.cpp and src/kernelfunctions.cu compiled for the
host, driven by oracle/ref_harness.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, tests/golden/make_golden.py and
bench.py's CPU-baseline leg; never by the product package.

Arrays use the reference's layout: DOFs and residuals are [var][basis][cell]
with var = (rho, rhou, rhov, rhoE), six P2 basis rows, and cells 0..T-1
owned followed by the ghost cells the reference adds on boundary edges.
"""
from __future__ import annotations

import ctypes as C
import os
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "librkdg_ref.so")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_lib = None


def reference_dir() -> str:
    """The reference checkout's multi_gpuRkdg directory: $RKDG_REF_DIR when
    set, else the REF_DIR default of oracle/Makefile (the recipe that
    compiles the reference's sources)."""
    env = os.environ.get("RKDG_REF_DIR")
    if env:
        return env
    with open(os.path.join(HERE, "Makefile")) as f:
        for line in f:
            if line.startswith("REF_DIR") and "?=" in line:
                return line.split("?=", 1)[1].strip()
    return ""


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"{LIB_PATH} not built (make -C oracle libref)")
        L = C.CDLL(LIB_PATH)
        L.rkdg_ref_open.restype = C.c_void_p
        L.rkdg_ref_open.argtypes = [C.c_char_p, C.c_char_p, _dp, C.c_int, C.c_char_p, C.c_int]
        L.rkdg_ref_close.argtypes = [C.c_void_p]
        L.rkdg_ref_sizes.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.rkdg_ref_set_farfield.argtypes = [C.c_void_p, _dp]
        L.rkdg_ref_init_freestream.argtypes = [C.c_void_p]
        L.rkdg_ref_get_geometry.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, _dp, _ip, _ip, _ip]
        L.rkdg_ref_get_tables.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, _dp, _dp]
        L.rkdg_ref_set_dofs.argtypes = [C.c_void_p, _dp]
        L.rkdg_ref_get_dofs.argtypes = [C.c_void_p, _dp]
        L.rkdg_ref_time_step.restype = C.c_double
        L.rkdg_ref_time_step.argtypes = [C.c_void_p]
        L.rkdg_ref_residual.argtypes = [C.c_void_p, _dp]
        L.rkdg_ref_save_old.argtypes = [C.c_void_p]
        L.rkdg_ref_stage.argtypes = [C.c_void_p, C.c_int, C.c_double]
        L.rkdg_ref_advance.argtypes = [C.c_void_p, C.c_int, _dp, _dp]
        L.rkdg_ref_set_threads.argtypes = [C.c_int]
        _lib = L
    return _lib


class RefCase:
    """One reference solver instance on a mesh (see ref_harness.cpp)."""

    def __init__(self, mesh, gamma=1.4, alpha_deg=0.0, mach=0.4, cfl=0.18, rhoref=1.0, pref=1.0,
                 threads_per_block=512, workdir=None):
        from rkdg_heter_calculate_b200 import meshgen

        self._tmp = None
        if workdir is None:
            self._tmp = tempfile.TemporaryDirectory(prefix="rkdg_ref_")
            workdir = self._tmp.name
        conf = meshgen.write_reference_format(mesh, workdir)
        params = np.array([gamma, alpha_deg, mach, cfl, rhoref, pref], dtype=np.float64)
        err = C.create_string_buffer(512)
        h = lib().rkdg_ref_open(workdir.encode(), conf.encode(), params, threads_per_block, err, 512)
        if not h:
            raise RuntimeError("reference set-up failed: " + err.value.decode(errors="replace"))
        self.h = C.c_void_p(h)
        t = C.c_int()
        n = C.c_int()
        lib().rkdg_ref_sizes(self.h, C.byref(t), C.byref(n))
        self.tnum, self.num = t.value, n.value
        self.gamma = gamma

    def close(self):
        if getattr(self, "h", None):
            lib().rkdg_ref_close(self.h)
            self.h = None
        if self._tmp is not None:
            self._tmp.cleanup()
            self._tmp = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_farfield(self, state):
        lib().rkdg_ref_set_farfield(self.h, np.ascontiguousarray(state, dtype=np.float64))

    def init_freestream(self):
        lib().rkdg_ref_init_freestream(self.h)

    def geometry(self):
        n = self.num
        out = dict(area=np.zeros(n), perimeter=np.zeros(n), normal=np.zeros((6, n)),
                   mass=np.zeros((6, n)), bary=np.zeros((2, n)),
                   neighbour=np.zeros((3, n), np.int32), shared=np.zeros((3, n), np.int32),
                   flag=np.zeros(n, np.int32))
        lib().rkdg_ref_get_geometry(self.h, out["area"], out["perimeter"], out["normal"],
                                    out["mass"], out["bary"], out["neighbour"], out["shared"],
                                    out["flag"])
        return out

    def tables(self):
        n = self.num
        out = dict(vol_bf=np.zeros((42, n)), vol_bdf=np.zeros((84, n)), edge_bf=np.zeros((54, n)),
                   vol_w=np.zeros((7, n)), edge_w=np.zeros((9, n)), coeff=np.zeros((n, 36)))
        lib().rkdg_ref_get_tables(self.h, out["vol_bf"], out["vol_bdf"], out["edge_bf"],
                                  out["vol_w"], out["edge_w"], out["coeff"])
        return out

    def set_dofs(self, U):
        """U: (4, 6, T) owned cells (ghost rows are left zero)."""
        full = np.zeros((4, 6, self.num))
        full[:, :, : U.shape[2]] = U
        lib().rkdg_ref_set_dofs(self.h, np.ascontiguousarray(full))

    def dofs(self):
        out = np.zeros((4, 6, self.num))
        lib().rkdg_ref_get_dofs(self.h, out)
        return out[:, :, : self.tnum].copy()

    def time_step(self) -> float:
        return lib().rkdg_ref_time_step(self.h)

    def residual(self):
        out = np.zeros((4, 6, self.num))
        lib().rkdg_ref_residual(self.h, out)
        return out[:, :, : self.tnum].copy()

    def save_old(self):
        lib().rkdg_ref_save_old(self.h)

    def stage(self, i: int, dt: float):
        lib().rkdg_ref_stage(self.h, i, dt)

    def advance(self, nsteps: int):
        dts = np.zeros(nsteps)
        res = np.zeros(2 * nsteps)
        lib().rkdg_ref_advance(self.h, nsteps, dts, res)
        return dts, res.reshape(nsteps, 2)


def set_threads(n: int):
    lib().rkdg_ref_set_threads(int(n))
