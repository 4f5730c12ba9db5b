"""Flow diagnostics of the vortex cases, evaluated identically for any state (device or oracle).

teal's Taylor-Green run computes none (run/taylor_green_vortex/run.c:23-59); these are the
volume-weighted averages the precision form reports its error on:
    kinetic energy  = sum(V * rho |u|^2 / 2) / sum(V)
    enstrophy       = sum(V * rho |curl u|^2 / 2) / sum(V)
with curl u from the least-squares gradient of the velocity (equations_gradient).
"""

import numpy as np


def kinetic_energy(primitive, volume):
    p = np.asarray(primitive)
    v = np.asarray(volume)[: p.shape[0]]
    return float((v * 0.5 * p[:, 0] * (p[:, 1:4] ** 2).sum(1)).sum() / v.sum())


def enstrophy(primitive, gradient, volume):
    """gradient: [cells][5][3] as teal stores it (velocity rows 1..3)."""
    p = np.asarray(primitive)
    g = np.asarray(gradient)
    n = g.shape[0]
    v = np.asarray(volume)[:n]
    du = g[:, 1:4, :]  # du[i][j] = d u_i / d x_j
    wx = du[:, 2, 1] - du[:, 1, 2]
    wy = du[:, 0, 2] - du[:, 2, 0]
    wz = du[:, 1, 0] - du[:, 0, 1]
    return float((v * 0.5 * p[:n, 0] * (wx**2 + wy**2 + wz**2)).sum() / v.sum())
