"""Shared test utilities: reference-basis projections and comparisons.

Test infrastructure; imports the oracle (the checker) freely.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from rkdg_heter_calculate_b200 import meshgen, vortex  # noqa: E402


def reference_basis_eval(coeff, mesh, X, Y, nb):
    """Values (T, Q, nb) of the reference's per-element basis (coefficients
    on 1, dx, dy, dx^2, dxdy, dy^2 about the barycentre) at points (T, Q)."""
    c = mesh.coords()
    xc = c[:, :, 0].mean(axis=1)[:, None]
    yc = c[:, :, 1].mean(axis=1)[:, None]
    dx, dy = X - xc, Y - yc
    mono = np.stack([np.ones_like(dx), dx, dy, dx * dx, dx * dy, dy * dy], axis=-1)  # (T,Q,6)
    return np.einsum("tqj,tij->tqi", mono, coeff[:, :nb, :])


def project_reference(mesh, func, coeff, nb, n=6):
    """L2 projection of func onto the reference basis: (4, nb, T)."""
    xi, eta, w = vortex.triangle_rule(n)
    X, Y = vortex.physical_points(mesh, xi, eta)
    phi = reference_basis_eval(coeff, mesh, X, Y, nb)  # (T,Q,nb)
    vals = func(X, Y)  # (4,T,Q)
    num = np.einsum("vtq,q,tqi->vit", vals, w, phi)
    den = np.einsum("q,tqi->it", w, phi * phi)
    return num / den[None]


def rel_err(a, b):
    """max |a-b| / max |b| per variable (normwise relative error)."""
    a = np.asarray(a)
    b = np.asarray(b)
    out = []
    for v in range(a.shape[0]):
        s = np.abs(b[v]).max()
        out.append(np.abs(a[v] - b[v]).max() / (s if s > 0 else 1.0))
    return max(out)


def vortex_state(mesh, coeff, nb, beta=5.0, uinf=1.0, vinf=1.0, gamma=1.4):
    return project_reference(mesh, lambda X, Y: vortex.exact(X, Y, 0.0, beta, gamma, uinf, vinf),
                             coeff, nb)


def perturbed_state(mesh, coeff, nb, base, amp=0.05, seed=0):
    """A smooth non-trivial state: base state plus a few sine modes."""
    def f(X, Y):
        r = base[0] * (1 + amp * np.sin(0.7 * X + 0.3) * np.cos(0.5 * Y))
        u = base[1] / base[0] + amp * np.cos(0.4 * X - 0.6 * Y)
        v = base[2] / base[0] + amp * np.sin(0.3 * X + 0.8 * Y)
        p = (base[3] - 0.5 * (base[1] ** 2 + base[2] ** 2) / base[0]) * 0.4 * (1 + amp * np.cos(0.2 * X * Y))
        return np.stack([r, r * u, r * v, p / 0.4 + 0.5 * r * (u * u + v * v)])
    return project_reference(mesh, f, coeff, nb)
