"""Flow diagnostics on downloaded states (host, numpy): volume-weighted kinetic
energy and enstrophy of a curvilinear block, and per-field error norms.

Volumes are 1/aj; velocity gradients use the same node-centred central
differences and metric transform as Compute_eddy_viscosity_LES (les.c:1533-1540)
on the interior nodes.
"""
from __future__ import annotations

import numpy as np


def _interior(a):
    return a[1:-1, 1:-1, 1:-1]


def kinetic_energy(q: np.ndarray, aj: np.ndarray) -> float:
    """sum(0.5 |rho u|^2 / rho / aj) / sum(1 / aj) over interior nodes."""
    rho = _interior(q[..., 0])
    m2 = sum(_interior(q[..., a]) ** 2 for a in (1, 2, 3))
    vol = 1.0 / _interior(aj)
    return float(np.sum(0.5 * m2 / rho * vol) / np.sum(vol))


def enstrophy(q: np.ndarray, csi: np.ndarray, eta: np.ndarray, zet: np.ndarray, aj: np.ndarray) -> float:
    """sum(0.5 rho |curl u|^2 / aj) / sum(1 / aj) over interior nodes."""
    u = [q[..., a] / q[..., 0] for a in (1, 2, 3)]

    def dc(f):  # d/dxi, d/deta, d/dzeta on interior nodes (axes: k, j, i)
        return (0.5 * (f[1:-1, 1:-1, 2:] - f[1:-1, 1:-1, :-2]),
                0.5 * (f[1:-1, 2:, 1:-1] - f[1:-1, :-2, 1:-1]),
                0.5 * (f[2:, 1:-1, 1:-1] - f[:-2, 1:-1, 1:-1]))

    ajc = _interior(aj)
    m = [_interior(csi), _interior(eta), _interior(zet)]
    g = []  # g[a][x] = d u_a / d x
    for a in range(3):
        d = dc(u[a])
        g.append([(d[0] * m[0][..., x] + d[1] * m[1][..., x] + d[2] * m[2][..., x]) * ajc for x in range(3)])
    wx = g[2][1] - g[1][2]
    wy = g[0][2] - g[2][0]
    wz = g[1][0] - g[0][1]
    vol = 1.0 / ajc
    rho = _interior(q[..., 0])
    return float(np.sum(0.5 * rho * (wx * wx + wy * wy + wz * wz) * vol) / np.sum(vol))


def field_errors(a: np.ndarray, ref: np.ndarray):
    """Per conserved field: relative L2 and relative Linf of a against ref."""
    l2, linf = [], []
    for f in range(a.shape[-1]):
        d = a[..., f] - ref[..., f]
        nr = float(np.linalg.norm(ref[..., f]))
        mr = float(np.abs(ref[..., f]).max())
        l2.append(float(np.linalg.norm(d)) / nr if nr else float(np.linalg.norm(d)))
        linf.append(float(np.abs(d).max()) / mr if mr else float(np.abs(d).max()))
    return l2, linf


def spectral_radius_max(q: np.ndarray, csi, eta, zet, aj, nvert, gamma: float = 1.4) -> float:
    """Host twin of the device CFL reduction: max over interior fluid nodes of
    aj * sum_d (|m_d . u| + c |m_d|)."""
    s = (slice(1, -1),) * 3
    r = q[s + (0,)]
    u, v, w = (q[s + (a,)] / r for a in (1, 2, 3))
    p = (gamma - 1) * (q[s + (4,)] - 0.5 * r * (u * u + v * v + w * w))
    c = np.sqrt(np.abs(gamma * p / r))
    lam = np.zeros_like(r)
    for m in (csi, eta, zet):
        mx, my, mz = m[s + (0,)], m[s + (1,)], m[s + (2,)]
        lam += np.abs(mx * u + my * v + mz * w) + c * np.sqrt(mx * mx + my * my + mz * mz)
    lam *= aj[s]
    lam[nvert[s] >= 0.1] = 0.0
    return float(lam.max())
