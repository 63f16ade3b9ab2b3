"""Host-side mirror of the reference solver's interface over the C ABI.

``CUDARkdgSolver`` keeps the method names and argument meanings of the
reference's ``CCUDARkdgSolver`` (multi_gpuRkdg/src/cudarkdgsolver.cu) and
``RkdgAdvance`` (src/rkdgadvance.cpp) so that code and tests written against
the reference's sequence read the same:

    reference                                   here
    ------------------------------------------  --------------------------------
    run + runNext (grid, geometry, H2D)          CUDARkdgSolver(mesh, ...)
    initRKDG                                     initRKDG()
    getTimeStep + dt read-back                   getTimeStep()
    calculateConVars .. calculateEdgeRHS         residual()   (one fused kernel)
    copy U -> U_old                              saveOld()
    rkdgStepOne/Two/Three                        rkdgStepOne/Two/Three(dt)
    RkdgAdvance::advance                         advance(nsteps, t_final)
    calculateResidual + residual read-back       the monitor returned by step()
    copyFreedomToHost                            copyFreedomToHost()
    outputSolution                               outputSolution(path)

Errors raise ``capi.RkdgError`` (the reference threw CMyException).
"""
from __future__ import annotations

import ctypes as C
import os
import math

import numpy as np

from . import capi

_FLUX = {"llf": capi.FLUX_LLF, "hllc": capi.FLUX_HLLC}
_LIM = {None: capi.LIMITER_NONE, "none": capi.LIMITER_NONE, "tvb": capi.LIMITER_TVB}
_PREC = {"fp64": capi.FP64, "fp32": capi.FP32, "fp32c": capi.FP32C}
_BASIS = {"reference": capi.BASIS_REFERENCE, "native": capi.BASIS_NATIVE}


def freestream_state(gamma=1.4, mach=0.4, alpha_deg=5.0, rhoref=1.0, pref=1.0):
    """Conservative far-field state as the reference builds it
    (src/rkdgadvance.cpp:31-34, src/cudarkdgsolver.cu:116)."""
    alpha = alpha_deg * math.atan(1.0) * 4 / 180
    ut = math.sqrt(gamma * pref / rhoref) * mach
    return (rhoref, rhoref * ut * math.cos(alpha), rhoref * ut * math.sin(alpha),
            0.5 * rhoref * ut * ut + pref / (gamma - 1))


def primitive_to_conservative(rho, u, v, p, gamma=1.4):
    return (rho, rho * u, rho * v, p / (gamma - 1) + 0.5 * rho * (u * u + v * v))


class CUDARkdgSolver:
    """One solve on one mesh, state resident in HBM (see module docstring)."""

    def __init__(self, mesh, order=2, nq=7, ng=3, flux="llf", limiter=None, rk=3,
                 precision="fp64", gamma=1.4, cfl=0.18, tvb_m=50.0, farfield=None,
                 reorder=True, n_owned=None):
        p = capi.default_params()
        p.order, p.nq, p.ng = order, nq, ng
        p.flux = _FLUX[flux]
        p.limiter = _LIM[limiter]
        p.rk = rk
        p.precision = _PREC[precision]
        p.reorder = 1 if reorder else 0
        p.gamma, p.cfl, p.tvb_m = gamma, cfl, tvb_m
        if farfield is None:
            farfield = freestream_state(gamma)
        for i in range(4):
            p.farfield[i] = farfield[i]
        self.params = p
        self.nbasis = 3 if order == 1 else 6
        d, keep = capi.mesh_desc(mesh.vertices, mesh.tris, getattr(mesh, "neighbours", None),
                                 getattr(mesh, "bc", None))
        h = C.c_void_p()
        if n_owned is None:
            capi.check(capi.lib().rkdg_create(C.byref(d), C.byref(p), C.byref(h)))
        else:  # one partition of a decomposed mesh (see decomp.py)
            capi.check(capi.lib().rkdg_create_part(C.byref(d), C.byref(p), int(n_owned), C.byref(h)))
        self.h = h
        self.T = d.ntri

    # -- lifetime ----------------------------------------------------------
    def close(self):
        if getattr(self, "h", None):
            capi.check(capi.lib().rkdg_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def sizes(self):
        t = C.c_int32()
        nb = C.c_int32()
        by = C.c_size_t()
        capi.check(capi.lib().rkdg_get_sizes(self.h, C.byref(t), C.byref(nb), C.byref(by)))
        return t.value, nb.value, by.value

    def part_rows(self):
        """(all state rows, cell-mean rows) of 16 bytes per element."""
        a, b = C.c_int32(), C.c_int32()
        capi.check(capi.lib().rkdg_part_rows(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def stream(self) -> int:
        s = C.c_void_p()
        capi.check(capi.lib().rkdg_get_stream(self.h, C.byref(s)))
        return s.value or 0

    # -- state -------------------------------------------------------------
    def initRKDG(self):
        capi.check(capi.lib().rkdg_init_freestream(self.h))

    def setFreedom(self, U, basis="reference"):
        U = np.ascontiguousarray(U, dtype=np.float64)
        if U.shape != (4, self.nbasis, self.T):
            raise ValueError(f"state must be (4, {self.nbasis}, {self.T})")
        capi.check(capi.lib().rkdg_set_state(self.h, capi.dptr(U), self.T, _BASIS[basis]))

    def copyFreedomToHost(self, basis="reference"):
        out = np.zeros((4, self.nbasis, self.T))
        capi.check(capi.lib().rkdg_get_state(self.h, capi.dptr(out), self.T, _BASIS[basis]))
        return out

    # -- hot path ----------------------------------------------------------
    def residual(self, basis="reference"):
        out = np.zeros((4, self.nbasis, self.T))
        capi.check(capi.lib().rkdg_residual(self.h, capi.dptr(out), self.T, _BASIS[basis]))
        return out

    def getTimeStep(self) -> float:
        dt = C.c_double()
        capi.check(capi.lib().rkdg_compute_dt(self.h, C.byref(dt)))
        return dt.value

    def saveOld(self):
        capi.check(capi.lib().rkdg_save_old(self.h))

    def stage(self, s: int, dt: float):
        capi.check(capi.lib().rkdg_stage(self.h, s, dt))

    def rkdgStepOne(self, dt):
        self.stage(0, dt)

    def rkdgStepTwo(self, dt):
        self.stage(1, dt)

    def rkdgStepThree(self, dt):
        self.stage(2, dt)

    def limit(self):
        capi.check(capi.lib().rkdg_limit(self.h))

    def step(self, dt: float = 0.0):
        """One time step; returns (dt_used, (max|d rho_mean|, max|d rhoE_mean|))."""
        du = C.c_double()
        mon = np.zeros(2)
        capi.check(capi.lib().rkdg_step(self.h, dt, C.byref(du), capi.dptr(mon)))
        return du.value, mon

    def advance(self, nsteps: int, t_final: float = 0.0):
        """nsteps device-resident steps (stopping at t_final when > 0);
        returns (time reached, steps taken)."""
        t = C.c_double()
        n = C.c_int32()
        capi.check(capi.lib().rkdg_advance(self.h, nsteps, t_final, C.byref(t), C.byref(n)))
        return t.value, n.value

    def time_stage(self, s: int, reps: int = 20) -> float:
        """Mean device milliseconds per launch of stage s's fused kernel."""
        ms = C.c_double()
        capi.check(capi.lib().rkdg_time_stage(self.h, s, reps, C.byref(ms)))
        return ms.value

    def time(self):
        t = C.c_double()
        n = C.c_int32()
        capi.check(capi.lib().rkdg_get_time(self.h, C.byref(t), C.byref(n)))
        return t.value, n.value

    def set_time(self, t: float):
        capi.check(capi.lib().rkdg_set_time(self.h, t))

    def conservation_totals(self):
        out = np.zeros(4)
        capi.check(capi.lib().rkdg_conservation_totals(self.h, capi.dptr(out)))
        return out

    def setResidualLog(self, path):
        """Residual history file as the reference writes it (None closes it)."""
        capi.check(capi.lib().rkdg_set_residual_log(self.h, None if path is None else os.fsencode(path)))

    def checkpoint(self, path: str):
        """Writes the full state, time and step count (bitwise restart)."""
        capi.check(capi.lib().rkdg_checkpoint_save(self.h, os.fsencode(path)))

    def restore(self, path: str):
        """Restores a checkpoint written on the same mesh, order and precision."""
        capi.check(capi.lib().rkdg_checkpoint_load(self.h, os.fsencode(path)))

    def outputSolution(self, path: str):
        capi.check(capi.lib().rkdg_write_solution(self.h, path.encode()))
