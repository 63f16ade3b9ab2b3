"""Serving loop over the C ABI (rkdg_server_*).

A native request loop admits solve requests into a device pool sized by an
HBM budget and advances every solve in flight together (one launch per RK
stage over all their tiles, a CUDA graph whose tile list changes without
recapture).  Requests carry their own mesh, order (P1 or P2), final time,
far-field state and limiter flag; the precision, flux, RK scheme and CFL
number belong to the server.  States cross the boundary in the native
basis, [4][nbasis][T] in the caller's triangle order.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import capi
from .solver import _FLUX, _PREC

QUEUED, RUNNING, DONE, FAILED = 0, 1, 2, 3


@dataclass
class Result:
    id: int
    status: int
    state: np.ndarray | None
    submitted: float
    admitted: float
    completed: float
    steps: int

    @property
    def latency(self) -> float:
        return self.completed - self.submitted


def clock() -> float:
    """Seconds on the loop's steady clock (the clock of Result's times)."""
    return capi.lib().rkdg_server_clock()


class Server:
    def __init__(self, hbm_budget_bytes: int, max_slots: int = 64, precision="fp32", flux="hllc",
                 rk=3, gamma=1.4, cfl=0.2, tvb_m=0.4, farfield=None):
        p = capi.default_params()
        p.order, p.nq, p.ng = 2, 6, 3
        p.flux = _FLUX[flux]
        p.rk = rk
        p.precision = _PREC[precision]
        p.gamma, p.cfl, p.tvb_m = gamma, cfl, tvb_m
        if farfield is not None:
            for v in range(4):
                p.farfield[v] = float(farfield[v])
        h = C.c_void_p()
        capi.check(capi.lib().rkdg_server_create(C.byref(p), int(hbm_budget_bytes), int(max_slots),
                                                 C.byref(h)))
        self.h = h
        self.params = p
        self._shape = {}

    def close(self):
        if getattr(self, "h", None):
            capi.check(capi.lib().rkdg_server_destroy(self.h))
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, mesh, order: int, U0: np.ndarray, t_final: float, farfield=None,
               limiter: bool = False, flux=None) -> int:
        """Queues a solve; flux ("llf" / "hllc") defaults to the server's."""
        nb = 3 if order == 1 else 6
        T = int(mesh.tris.shape[0])
        U0 = np.ascontiguousarray(U0, dtype=np.float64)
        assert U0.shape == (4, nb, T), U0.shape
        d, keep = capi.mesh_desc(mesh.vertices, mesh.tris, getattr(mesh, "neighbours", None),
                                 getattr(mesh, "bc", None))
        far = None if farfield is None else np.ascontiguousarray(farfield, dtype=np.float64)
        rid = C.c_int64()
        fl = self.params.flux if flux is None else _FLUX[flux]
        capi.check(capi.lib().rkdg_server_submit_method(self.h, C.byref(d), int(order), capi.dptr(U0),
                                                        float(t_final),
                                                        capi.dptr(far) if far is not None else None,
                                                        int(bool(limiter)), fl, C.byref(rid)))
        del keep
        self._shape[rid.value] = (4, nb, T)
        return rid.value

    def wait(self, rid: int, timeout: float = -1.0) -> Result:
        shape = self._shape[rid]
        U = np.zeros(shape)
        times = np.zeros(3)
        st, steps = C.c_int32(), C.c_int32()
        rc = capi.lib().rkdg_server_wait(self.h, rid, float(timeout), C.byref(st), capi.dptr(U),
                                         capi.dptr(times), C.byref(steps))
        if st.value >= DONE:
            self._shape.pop(rid, None)
        capi.check(rc)
        return Result(rid, st.value, U if st.value == DONE else None, times[0], times[1], times[2],
                      steps.value)

    def status(self) -> dict:
        """Queued and in-flight counts; raises RkdgError once the loop has
        stopped on an error."""
        q, f = C.c_int32(), C.c_int32()
        capi.check(capi.lib().rkdg_server_status(self.h, C.byref(q), C.byref(f)))
        return {"queued": q.value, "in_flight": f.value}

    def inject_fault(self, after_chunks: int = 0):
        """Test support: the loop stops as on a failed CUDA call (nothing is
        done to the device)."""
        capi.check(capi.lib().rkdg_server_inject_fault(self.h, int(after_chunks)))

    def timing(self) -> dict:
        """Engine seconds uploading, retiring and stepping, and step chunks."""
        a, r, st = C.c_double(), C.c_double(), C.c_double()
        n = C.c_int64()
        capi.check(capi.lib().rkdg_server_timing(self.h, C.byref(a), C.byref(r), C.byref(st), C.byref(n)))
        return {"admit_s": a.value, "retire_s": r.value, "step_s": st.value, "chunks": n.value}

    def stats(self) -> dict:
        dof, busy = C.c_double(), C.c_double()
        done, cap = C.c_int64(), C.c_int64()
        peak = C.c_int32()
        capi.check(capi.lib().rkdg_server_stats(self.h, C.byref(dof), C.byref(busy), C.byref(done),
                                                C.byref(peak), C.byref(cap)))
        return {"dof_stage_updates": dof.value, "busy_seconds": busy.value, "completed": done.value,
                "peak_in_flight": peak.value, "capacity_elements": cap.value}
