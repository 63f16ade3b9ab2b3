"""Isentropic-vortex test problem (Shu's vortex): exact solution, L2
projection onto the native basis and L2 error, all in FP64 on the host.

Free stream (rho, u, v, p) = (1, u_inf, v_inf, 1); vortex of strength beta
centred at (5, 5) on the periodic square [0, 10]^2:

    du = -beta/(2 pi) (y - yc) exp((1 - r^2)/2),  dv = beta/(2 pi) (x - xc) exp((1 - r^2)/2)
    T  = 1 - (gamma - 1) beta^2 / (8 gamma pi^2) exp(1 - r^2),  rho = T^(1/(gamma-1)),  p = rho^gamma

The exact solution at time t is the initial state advected by (u_inf, v_inf)
with periodic images.  Projections and errors use a collapsed (Duffy)
Gauss-Legendre rule of n x n points on each triangle, exact to degree 2n-2.
"""
from __future__ import annotations

import math

import numpy as np

from . import capi


def exact(x, y, t=0.0, beta=5.0, gamma=1.4, uinf=1.0, vinf=1.0, L=10.0, xc=5.0, yc=5.0):
    """Conservative variables (4, ...) of the advected vortex at (x, y, t)."""
    dx = np.mod(x - uinf * t - xc + 0.5 * L, L) - 0.5 * L
    dy = np.mod(y - vinf * t - yc + 0.5 * L, L) - 0.5 * L
    r2 = dx * dx + dy * dy
    f = np.exp(0.5 * (1.0 - r2))
    u = uinf - beta / (2 * math.pi) * dy * f
    v = vinf + beta / (2 * math.pi) * dx * f
    T = 1.0 - (gamma - 1.0) * beta * beta / (8.0 * gamma * math.pi ** 2) * f * f
    rho = T ** (1.0 / (gamma - 1.0))
    p = rho ** gamma
    return np.stack([rho, rho * u, rho * v, p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v)])


def triangle_rule(n: int = 6):
    """Collapsed Gauss rule on the reference triangle: (xi, eta, w) with the
    weights normalised to sum to one (area average)."""
    g, w = np.polynomial.legendre.leggauss(n)
    s = 0.5 * (g + 1.0)
    ws = 0.5 * w
    U, V = np.meshgrid(s, s, indexing="ij")
    WU, WV = np.meshgrid(ws, ws, indexing="ij")
    xi = U.reshape(-1)
    eta = (V * (1.0 - U)).reshape(-1)
    wt = (WU * WV * (1.0 - U)).reshape(-1) * 2.0
    return xi, eta, wt


def physical_points(mesh, xi, eta):
    """(T, Q) coordinates x = v0 + xi (v1 - v0) + eta (v2 - v0)."""
    c = mesh.coords()
    a = c[:, 1] - c[:, 0]
    b = c[:, 2] - c[:, 0]
    X = c[:, 0, 0:1] + a[:, 0:1] * xi[None] + b[:, 0:1] * eta[None]
    Y = c[:, 0, 1:2] + a[:, 1:2] * xi[None] + b[:, 1:2] * eta[None]
    return X, Y


def project_native(mesh, func, nbasis: int, n: int = 6) -> np.ndarray:
    """L2 projection of func(x, y) -> (4, T, Q) onto the native basis:
    coefficients (4, nbasis, T) (the basis is orthonormal under the area average)."""
    xi, eta, w = triangle_rule(n)
    psi = capi.native_basis(nbasis, xi, eta)  # (Q, nb)
    X, Y = physical_points(mesh, xi, eta)
    vals = func(X, Y)  # (4, T, Q)
    return np.einsum("vtq,q,qi->vit", vals, w, psi)


def l2_error(mesh, U_native: np.ndarray, func, var: int = 0, n: int = 6) -> float:
    """RMS over the domain of (u_h - func)[var]: sqrt(sum_e int_e err^2 / area)."""
    nb = U_native.shape[1]
    xi, eta, w = triangle_rule(n)
    psi = capi.native_basis(nb, xi, eta)
    X, Y = physical_points(mesh, xi, eta)
    uh = np.einsum("it,qi->tq", U_native[var], psi)
    ex = func(X, Y)[var]
    area = mesh.areas()
    err2 = (area[:, None] * w[None] * (uh - ex) ** 2).sum()
    return float(math.sqrt(err2 / area.sum()))
