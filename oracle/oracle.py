"""ctypes front-end of oracle/librkdg_oracle.so, the plain-C restatement of
the reference RKDG algorithm (rkdg_oracle.c).

TEST INFRASTRUCTURE ONLY: the checker used by tests/, by the smoke check in
__graft_entry__.py and by bench.py's CPU leg.  The product never imports it.

State/residual layout: (4, Nb, T) in the reference's per-element basis.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librkdg_oracle.so")

LLF, HLLC = 0, 1
LIMITER_NONE, LIMITER_TVB = 0, 1

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


class Params(C.Structure):
    _fields_ = [("order", C.c_int), ("nq", C.c_int), ("ng", C.c_int), ("flux", C.c_int),
                ("limiter", C.c_int), ("rk", C.c_int), ("tvb_m", C.c_double),
                ("gamma", C.c_double), ("cfl", C.c_double), ("farfield", C.c_double * 4)]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE, "liboracle"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.oracle_create.restype = C.c_void_p
        L.oracle_create.argtypes = [C.c_int, _dp, _ip, _ip, C.POINTER(Params)]
        L.oracle_destroy.argtypes = [C.c_void_p]
        L.oracle_nbasis.restype = C.c_int
        L.oracle_nbasis.argtypes = [C.c_void_p]
        L.oracle_set_threads.argtypes = [C.c_int]
        L.oracle_get_basis.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, _dp]
        L.oracle_set_state.argtypes = [C.c_void_p, _dp]
        L.oracle_get_state.argtypes = [C.c_void_p, _dp]
        L.oracle_save_old.argtypes = [C.c_void_p]
        L.oracle_residual.argtypes = [C.c_void_p, _dp]
        L.oracle_time_step.restype = C.c_double
        L.oracle_time_step.argtypes = [C.c_void_p]
        L.oracle_stage.argtypes = [C.c_void_p, C.c_int, C.c_double]
        L.oracle_limit.restype = C.c_int
        L.oracle_limit.argtypes = [C.c_void_p]
        L.oracle_step.restype = C.c_double
        L.oracle_step.argtypes = [C.c_void_p, C.c_double, _dp]
        L.oracle_eval.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _dp]
        _lib = L
    return _lib


def set_threads(n: int):
    lib().oracle_set_threads(int(n))


class Oracle:
    """One oracle solver on a mesh (rkdg_heter_calculate_b200.meshgen.Mesh)."""

    def __init__(self, mesh, order=2, nq=7, ng=3, flux=LLF, limiter=LIMITER_NONE, rk=3,
                 tvb_m=50.0, gamma=1.4, cfl=0.18, farfield=(1.0, 0.0, 0.0, 2.5)):
        p = Params(order, nq, ng, flux, limiter, rk, tvb_m, gamma, cfl,
                   (C.c_double * 4)(*farfield))
        xy = np.ascontiguousarray(mesh.coords().reshape(-1), dtype=np.float64)
        nbr = np.ascontiguousarray(mesh.neighbours.reshape(-1), dtype=np.int32)
        bc = np.ascontiguousarray(mesh.bc.reshape(-1).astype(np.int32))
        h = lib().oracle_create(mesh.ntri, xy, nbr, bc, C.byref(p))
        if not h:
            raise ValueError("oracle_create rejected the mesh/parameters")
        self.h = C.c_void_p(h)
        self.T = mesh.ntri
        self.nb = lib().oracle_nbasis(self.h)
        self.params = p

    def close(self):
        if getattr(self, "h", None):
            lib().oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def basis(self):
        T = self.T
        out = dict(coeff=np.zeros((T, 6, 6)), mass=np.zeros((T, 6)), area=np.zeros(T),
                   perimeter=np.zeros(T), normal=np.zeros((T, 3, 2)))
        lib().oracle_get_basis(self.h, out["coeff"], out["mass"], out["area"], out["perimeter"],
                               out["normal"])
        return out

    def set_state(self, U):
        U = np.ascontiguousarray(U, dtype=np.float64)
        assert U.shape == (4, self.nb, self.T)
        lib().oracle_set_state(self.h, U)

    def state(self):
        out = np.zeros((4, self.nb, self.T))
        lib().oracle_get_state(self.h, out)
        return out

    def save_old(self):
        lib().oracle_save_old(self.h)

    def residual(self):
        out = np.zeros((4, self.nb, self.T))
        lib().oracle_residual(self.h, out)
        return out

    def time_step(self) -> float:
        return lib().oracle_time_step(self.h)

    def stage(self, s: int, dt: float):
        lib().oracle_stage(self.h, s, dt)

    def limit(self) -> int:
        return lib().oracle_limit(self.h)

    def step(self, dt: float = -1.0):
        mon = np.zeros(2)
        dt = lib().oracle_step(self.h, dt, mon)
        return dt, mon

    def eval(self, l1, l2):
        l1 = np.ascontiguousarray(l1, dtype=np.float64)
        l2 = np.ascontiguousarray(l2, dtype=np.float64)
        out = np.zeros((4, l1.size, self.T))
        lib().oracle_eval(self.h, l1.size, l1, l2, out)
        return out
