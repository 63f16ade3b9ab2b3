"""B200-native (sm_100a) RKDG residual and time-step path for the 2D Euler
equations on unstructured triangles, behind the C ABI of include/rkdg.h.

    from rkdg_heter_calculate_b200 import CUDARkdgSolver, meshgen

The CUDA library (librkdg.so, built in-tree for sm_100a) is the only
compute path; importing this package does not load it, the first solver
call does, and fails loudly if it or a B200 is missing.
"""
from .capi import RkdgError, lib  # noqa: F401
from .solver import CUDARkdgSolver, freestream_state, primitive_to_conservative  # noqa: F401

__all__ = ["CUDARkdgSolver", "RkdgError", "freestream_state", "primitive_to_conservative", "lib"]
