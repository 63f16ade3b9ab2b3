"""ctypes bindings of librkdg.so (include/rkdg.h).

The library is loaded from this package directory only (built in-tree by
``python -m rkdg_heter_calculate_b200.build``); there is no fallback: every
entry point raises if the library or a CUDA device is missing.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "librkdg.so")

RKDG_OK = 0
RKDG_ERR_INVALID, RKDG_ERR_CUDA, RKDG_ERR_NOMEM, RKDG_ERR_STATE = 1, 2, 3, 4
RKDG_ERR_NODEVICE, RKDG_ERR_IO, RKDG_ERR_BUSY = 5, 6, 7
ERRORS = {1: "INVALID", 2: "CUDA", 3: "NOMEM", 4: "STATE", 5: "NODEVICE", 6: "IO", 7: "BUSY"}
FLUX_LLF, FLUX_HLLC = 0, 1
LIMITER_NONE, LIMITER_TVB = 0, 1
FP64, FP32, FP32C = 0, 1, 2
BASIS_REFERENCE, BASIS_NATIVE = 0, 1
BC_FARFIELD, BC_OUTFLOW, BC_REFLECTION = 1, 2, 3


class RkdgError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"rkdg error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


class MeshDesc(C.Structure):
    _fields_ = [("ntri", C.c_int32), ("nvert", C.c_int32), ("vertices", C.POINTER(C.c_double)),
                ("tri_vertex", C.POINTER(C.c_int32)), ("tri_neighbour", C.POINTER(C.c_int32)),
                ("bc", C.POINTER(C.c_int8))]


class Params(C.Structure):
    _fields_ = [("order", C.c_int32), ("nq", C.c_int32), ("ng", C.c_int32), ("flux", C.c_int32),
                ("limiter", C.c_int32), ("rk", C.c_int32), ("precision", C.c_int32),
                ("reorder", C.c_int32), ("gamma", C.c_double), ("cfl", C.c_double),
                ("tvb_m", C.c_double), ("farfield", C.c_double * 4)]


_lib = None
_dp = C.POINTER(C.c_double)


def lib():
    """Loads librkdg.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run python -m rkdg_heter_calculate_b200.build")
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        sig = {
            "rkdg_last_error": (C.c_char_p, []),
            "rkdg_default_params": (None, [C.POINTER(Params)]),
            "rkdg_create": (C.c_int, [C.POINTER(MeshDesc), C.POINTER(Params), C.POINTER(vp)]),
            "rkdg_destroy": (C.c_int, [vp]),
            "rkdg_get_sizes": (C.c_int, [vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_size_t)]),
            "rkdg_get_stream": (C.c_int, [vp, C.POINTER(vp)]),
            "rkdg_init_freestream": (C.c_int, [vp]),
            "rkdg_set_state": (C.c_int, [vp, _dp, C.c_int32, C.c_int32]),
            "rkdg_get_state": (C.c_int, [vp, _dp, C.c_int32, C.c_int32]),
            "rkdg_residual": (C.c_int, [vp, _dp, C.c_int32, C.c_int32]),
            "rkdg_compute_dt": (C.c_int, [vp, _dp]),
            "rkdg_save_old": (C.c_int, [vp]),
            "rkdg_stage": (C.c_int, [vp, C.c_int32, C.c_double]),
            "rkdg_limit": (C.c_int, [vp]),
            "rkdg_step": (C.c_int, [vp, C.c_double, _dp, _dp]),
            "rkdg_advance": (C.c_int, [vp, C.c_int32, C.c_double, _dp, C.POINTER(C.c_int32)]),
            "rkdg_get_time": (C.c_int, [vp, _dp, C.POINTER(C.c_int32)]),
            "rkdg_time_stage": (C.c_int, [vp, C.c_int32, C.c_int32, _dp]),
            "rkdg_set_time": (C.c_int, [vp, C.c_double]),
            "rkdg_conservation_totals": (C.c_int, [vp, _dp]),
            "rkdg_write_solution": (C.c_int, [vp, C.c_char_p]),
            "rkdg_read_mesh": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(MeshDesc)]),
            "rkdg_free_mesh": (None, [C.POINTER(MeshDesc)]),
            "rkdg_native_basis": (C.c_int, [C.c_int32, C.c_int32, _dp, _dp, _dp]),
            "rkdg_build_connectivity": (C.c_int, [C.POINTER(MeshDesc), C.POINTER(C.c_int32),
                                                  C.POINTER(C.c_int8), C.POINTER(C.c_int8)]),
            "rkdg_locality_order": (C.c_int, [C.POINTER(MeshDesc), C.POINTER(C.c_int32)]),
            "rkdg_conservation_totals_noalloc": (C.c_int, [C.c_int32, C.c_void_p, C.c_int32,
                                                           C.c_void_p, C.c_void_p, C.c_void_p]),
            "rkdg_batch_create": (C.c_int, [C.c_int32, C.POINTER(MeshDesc), C.POINTER(C.c_int32),
                                            _dp, C.POINTER(Params), C.POINTER(vp)]),
            "rkdg_batch_destroy": (C.c_int, [vp]),
            "rkdg_batch_set_state": (C.c_int, [vp, C.c_int32, _dp, C.c_int32]),
            "rkdg_batch_get_state": (C.c_int, [vp, C.c_int32, _dp, C.c_int32]),
            "rkdg_batch_advance": (C.c_int, [vp, C.c_int32, _dp, _dp, C.POINTER(C.c_int32)]),
            "rkdg_batch_set_time": (C.c_int, [vp, C.c_int32, C.c_double]),
            "rkdg_batch_autotune": (C.c_int, [vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                              C.POINTER(C.c_int32)]),
            "rkdg_batch_set_tile": (C.c_int, [vp, C.c_int32]),
            "rkdg_batch_set_shape": (C.c_int, [vp, C.c_int32, C.c_int32]),
            "rkdg_batch_time_stage": (C.c_int, [vp, C.c_int32, C.c_int32, _dp]),
            "rkdg_batch_get_sizes": (C.c_int, [vp, C.POINTER(C.c_int64), C.POINTER(C.c_int32),
                                               C.POINTER(C.c_size_t)]),
            "rkdg_batch_get_stream": (C.c_int, [vp, C.POINTER(vp)]),
            "rkdg_server_create": (C.c_int, [C.POINTER(Params), C.c_size_t, C.c_int32, C.POINTER(vp)]),
            "rkdg_server_destroy": (C.c_int, [vp]),
            "rkdg_server_submit": (C.c_int, [vp, C.POINTER(MeshDesc), C.c_int32, _dp, C.c_double, _dp,
                                             C.c_int32, C.POINTER(C.c_int64)]),
            "rkdg_server_submit_method": (C.c_int, [vp, C.POINTER(MeshDesc), C.c_int32, _dp, C.c_double, _dp,
                                                    C.c_int32, C.c_int32, C.POINTER(C.c_int64)]),
            "rkdg_server_wait": (C.c_int, [vp, C.c_int64, C.c_double, C.POINTER(C.c_int32), _dp, _dp,
                                           C.POINTER(C.c_int32)]),
            "rkdg_server_stats": (C.c_int, [vp, _dp, _dp, C.POINTER(C.c_int64), C.POINTER(C.c_int32),
                                            C.POINTER(C.c_int64)]),
            "rkdg_server_clock": (C.c_double, []),
            "rkdg_create_part": (C.c_int, [C.POINTER(MeshDesc), C.POINTER(Params), C.c_int32, C.POINTER(vp)]),
            "rkdg_part_rows": (C.c_int, [vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
            "rkdg_gather_rows": (C.c_int, [vp, vp, C.c_int32, C.c_int32, vp]),
            "rkdg_scatter_rows": (C.c_int, [vp, vp, C.c_int32, C.c_int32, vp]),
            "rkdg_sync": (C.c_int, [vp]),
            "rkdg_part_set_final_time": (C.c_int, [vp, C.c_double]),
            "rkdg_part_wave": (C.c_int, [vp, vp, C.c_int32]),
            "rkdg_part_begin_step": (C.c_int, [vp]),
            "rkdg_part_stage": (C.c_int, [vp, C.c_int32]),
            "rkdg_part_stage_begin": (C.c_int, [vp, C.c_int32]),
            "rkdg_part_stage_end": (C.c_int, [vp, C.c_int32]),
            "rkdg_part_limit": (C.c_int, [vp]),
            "rkdg_part_time": (C.c_int, [vp, _dp, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
            "rkdg_server_status": (C.c_int, [vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
            "rkdg_server_timing": (C.c_int, [vp, _dp, _dp, _dp, C.POINTER(C.c_int64)]),
            "rkdg_server_inject_fault": (C.c_int, [vp, C.c_int32]),
            "rkdg_checkpoint_save": (C.c_int, [vp, C.c_char_p]),
            "rkdg_checkpoint_load": (C.c_int, [vp, C.c_char_p]),
            "rkdg_set_residual_log": (C.c_int, [vp, C.c_char_p]),
            "rkdg_wait_selftest": (C.c_int, [C.c_double, C.POINTER(C.c_int32), _dp]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int):
    if rc != RKDG_OK:
        raise RkdgError(rc, lib().rkdg_last_error().decode(errors="replace"))


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


def default_params() -> Params:
    p = Params()
    lib().rkdg_default_params(C.byref(p))
    return p


def native_basis(nbasis: int, xi, eta) -> np.ndarray:
    xi = np.ascontiguousarray(xi, dtype=np.float64)
    eta = np.ascontiguousarray(eta, dtype=np.float64)
    out = np.zeros((xi.size, nbasis))
    check(lib().rkdg_native_basis(nbasis, xi.size, dptr(xi), dptr(eta), dptr(out)))
    return out


def mesh_desc(vertices, tris, neighbours=None, bc=None):
    """MeshDesc over numpy arrays; returns (desc, keep-alive list)."""
    verts = np.ascontiguousarray(vertices, dtype=np.float64).reshape(-1)
    tv = np.ascontiguousarray(tris, dtype=np.int32).reshape(-1)
    d = MeshDesc()
    d.ntri = tv.size // 3
    d.nvert = verts.size // 2
    d.vertices = verts.ctypes.data_as(C.POINTER(C.c_double))
    d.tri_vertex = tv.ctypes.data_as(C.POINTER(C.c_int32))
    keep = [verts, tv]
    if neighbours is not None:
        nb = np.ascontiguousarray(neighbours, dtype=np.int32).reshape(-1)
        d.tri_neighbour = nb.ctypes.data_as(C.POINTER(C.c_int32))
        keep.append(nb)
    if bc is not None:
        b = np.ascontiguousarray(bc, dtype=np.int8).reshape(-1)
        d.bc = b.ctypes.data_as(C.POINTER(C.c_int8))
        keep.append(b)
    return d, keep


def build_connectivity(vertices, tris, neighbours=None, bc=None):
    """Host-only connectivity as rkdg_create builds it: (neighbour, shared, bc)."""
    d, keep = mesh_desc(vertices, tris, neighbours, bc)
    T = d.ntri
    nb = np.zeros((T, 3), np.int32)
    sh = np.zeros((T, 3), np.int8)
    tags = np.zeros((T, 3), np.int8)
    check(lib().rkdg_build_connectivity(C.byref(d), nb.ctypes.data_as(C.POINTER(C.c_int32)),
                                        sh.ctypes.data_as(C.POINTER(C.c_int8)),
                                        tags.ctypes.data_as(C.POINTER(C.c_int8))))
    return nb, sh, tags


def locality_order(vertices, tris, neighbours=None):
    d, keep = mesh_desc(vertices, tris, neighbours)
    perm = np.zeros(d.ntri, np.int32)
    check(lib().rkdg_locality_order(C.byref(d), perm.ctypes.data_as(C.POINTER(C.c_int32))))
    return perm


def read_mesh(base_dir: str, mesh_conf: str):
    """Reads the reference's mesh file set: (vertices, tris, neighbours or None)."""
    d = MeshDesc()
    check(lib().rkdg_read_mesh(base_dir.encode(), mesh_conf.encode(), C.byref(d)))
    try:
        V = np.ctypeslib.as_array(d.vertices, shape=(d.nvert * 2,)).reshape(-1, 2).copy()
        T = np.ctypeslib.as_array(d.tri_vertex, shape=(d.ntri * 3,)).reshape(-1, 3).copy()
        N = None
        if d.tri_neighbour:
            N = np.ctypeslib.as_array(d.tri_neighbour, shape=(d.ntri * 3,)).reshape(-1, 3).copy()
    finally:
        lib().rkdg_free_mesh(C.byref(d))
    return V, T, N
