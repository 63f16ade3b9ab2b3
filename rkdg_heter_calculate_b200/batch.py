"""Batched independent solves over the C ABI (rkdg_batch_*).

Many solves on meshes of uneven size and mixed order share one packed
element space; every RK stage of all of them is one launch of the
tile-staged kernel, each solve keeps its own dt, time and final time, and
the whole step is one CUDA graph.  States cross the boundary in the native
basis, [4][nbasis][T] per solve in its caller's triangle order.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi
from .solver import _FLUX, _PREC


class Batch:
    def __init__(self, meshes, orders, precision="fp32", flux="hllc", rk=3, nq=6, gamma=1.4,
                 cfl=0.2, farfields=None, reorder=True):
        p = capi.default_params()
        p.reorder = 1 if reorder else 0
        p.order = 2
        p.nq = nq
        p.ng = 3
        p.flux = _FLUX[flux]
        p.rk = rk
        p.precision = _PREC[precision]
        p.gamma, p.cfl = gamma, cfl
        S = len(meshes)
        descs = (capi.MeshDesc * S)()
        self._keep = []
        for i, m in enumerate(meshes):
            d, keep = capi.mesh_desc(m.vertices, m.tris, getattr(m, "neighbours", None),
                                     getattr(m, "bc", None))
            descs[i] = d
            self._keep.append(keep)
        self.orders = np.ascontiguousarray(orders, dtype=np.int32)
        self.T = [int(m.tris.shape[0]) for m in meshes]
        far = None
        if farfields is not None:
            far = np.ascontiguousarray(farfields, dtype=np.float64).reshape(S, 4)
        h = C.c_void_p()
        capi.check(capi.lib().rkdg_batch_create(
            S, descs, self.orders.ctypes.data_as(C.POINTER(C.c_int32)),
            capi.dptr(far) if far is not None else None, C.byref(p), C.byref(h)))
        self.h = h
        self.S = S

    def close(self):
        if getattr(self, "h", None):
            capi.check(capi.lib().rkdg_batch_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def nbasis(self, s):
        return 3 if self.orders[s] == 1 else 6

    def set_state(self, s, U):
        U = np.ascontiguousarray(U, dtype=np.float64)
        assert U.shape == (4, self.nbasis(s), self.T[s])
        capi.check(capi.lib().rkdg_batch_set_state(self.h, s, capi.dptr(U), self.T[s]))

    def state(self, s):
        out = np.zeros((4, self.nbasis(s), self.T[s]))
        capi.check(capi.lib().rkdg_batch_get_state(self.h, s, capi.dptr(out), self.T[s]))
        return out

    def set_time(self, s, t):
        capi.check(capi.lib().rkdg_batch_set_time(self.h, s, t))

    def advance(self, nsteps, t_final=None):
        tf = None
        if t_final is not None:
            tf = np.ascontiguousarray(t_final, dtype=np.float64)
        t = np.zeros(self.S)
        n = np.zeros(self.S, dtype=np.int32)
        capi.check(capi.lib().rkdg_batch_advance(self.h, nsteps, capi.dptr(tf) if tf is not None else None,
                                                 capi.dptr(t), n.ctypes.data_as(C.POINTER(C.c_int32))))
        return t, n

    def autotune(self):
        """Times the candidate launch shapes; returns (CTAs, tile order, tile size)."""
        c, o, t = C.c_int32(), C.c_int32(), C.c_int32()
        capi.check(capi.lib().rkdg_batch_autotune(self.h, C.byref(c), C.byref(o), C.byref(t)))
        return c.value, o.value, t.value

    def set_tile(self, tile):
        capi.check(capi.lib().rkdg_batch_set_tile(self.h, int(tile)))

    def set_shape(self, ctas, tile_order=0):
        capi.check(capi.lib().rkdg_batch_set_shape(self.h, ctas, tile_order))

    def time_stage(self, s=1, reps=10):
        ms = C.c_double()
        capi.check(capi.lib().rkdg_batch_time_stage(self.h, s, reps, C.byref(ms)))
        return ms.value

    def sizes(self):
        e = C.c_int64()
        t = C.c_int32()
        b = C.c_size_t()
        capi.check(capi.lib().rkdg_batch_get_sizes(self.h, C.byref(e), C.byref(t), C.byref(b)))
        return e.value, t.value, b.value

    def stream(self):
        s = C.c_void_p()
        capi.check(capi.lib().rkdg_batch_get_stream(self.h, C.byref(s)))
        return s.value or 0
