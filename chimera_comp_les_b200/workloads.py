"""Seeded synthetic inputs (grids and initial states) for the RHS/RK path.

No dataset is involved: every workload is generated here from a formula and
a seed.  Arrays are in the reference's natural node order, AoS:
coordinates (mz, my, mx, 3), conserved state (mz, my, mx, 5) with
components (rho, rho*u, rho*v, rho*w, rho*E).

Periodic sizing follows the reference's DMDA convention: N unique points per
direction are stored as m = N + 2 nodes, node i at x = (i - 1) * L / N, so
node 0 is the image of node m-2 and node m-1 the image of node 1
(rhs.c:1107-1227).
"""
from __future__ import annotations

import math

import numpy as np


def periodic_grid(n, length, amp: float = 0.0) -> np.ndarray:
    """Curvilinear periodic box.  n, length: int/float or 3-tuples (x, y, z).

    amp > 0 perturbs the nodes cyclically, x_i += amp*sin(xi_j)*sin(xi_k) with
    xi = 2*pi*x/L, so the metrics are non-trivial but stay periodic.
    """
    ns = (n, n, n) if np.isscalar(n) else tuple(n)
    ls = (length, length, length) if np.isscalar(length) else tuple(length)
    ax = [(np.arange(ns[d] + 2) - 1.0) * (ls[d] / ns[d]) for d in range(3)]
    z, y, x = np.meshgrid(ax[2], ax[1], ax[0], indexing="ij")
    if amp:
        sx, sy, sz = (2 * math.pi * x / ls[0], 2 * math.pi * y / ls[1], 2 * math.pi * z / ls[2])
        x, y, z = (x + amp * np.sin(sy) * np.sin(sz), y + amp * np.sin(sz) * np.sin(sx),
                   z + amp * np.sin(sx) * np.sin(sy))
    return np.ascontiguousarray(np.stack([x, y, z], axis=-1))


def conserved(rho, u, v, w, p, gamma: float) -> np.ndarray:
    e = p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v + w * w)
    return np.ascontiguousarray(np.stack([rho, rho * u, rho * v, rho * w, e], axis=-1))


def tgv_state(coords: np.ndarray, gamma: float = 1.4, ma: float = 0.1, p0: float = 100.0) -> np.ndarray:
    """Compressible Taylor-Green vortex with the reference's scaling
    (rhs.c:278-294): rho = gamma*p*Ma^2 and the momentum set to the velocity
    profile itself."""
    x, y, z = coords[..., 0], coords[..., 1], coords[..., 2]
    p = p0 + (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2.0) / 16.0
    rho = gamma * p * ma * ma
    ru = np.sin(x) * np.cos(y) * np.cos(z)
    rv = -np.cos(x) * np.sin(y) * np.cos(z)
    rw = np.zeros_like(x)
    e = p / (gamma - 1.0) + 0.5 * (ru * ru + rv * rv + rw * rw) / rho
    return np.ascontiguousarray(np.stack([rho, ru, rv, rw, e], axis=-1))


def vortex_state(coords: np.ndarray, gamma: float = 1.4, beta: float = 5.0, center=(5.0, 5.0),
                 uinf=(1.0, 1.0, 0.0)) -> np.ndarray:
    """Isentropic (Shu) vortex, uniform in z, on a free stream rho = p = 1."""
    x, y = coords[..., 0], coords[..., 1]
    dx, dy = x - center[0], y - center[1]
    r2 = dx * dx + dy * dy
    f = beta / (2 * math.pi) * np.exp(0.5 * (1.0 - r2))
    u = uinf[0] - f * dy
    v = uinf[1] + f * dx
    w = np.full_like(x, uinf[2])
    t = 1.0 - (gamma - 1.0) * beta * beta / (8.0 * gamma * math.pi ** 2) * np.exp(1.0 - r2)
    rho = t ** (1.0 / (gamma - 1.0))
    p = rho ** gamma
    return conserved(rho, u, v, w, p, gamma)


def random_smooth_state(shape, seed: int, gamma: float = 1.4, amp: float = 0.05, periodic: bool = True) -> np.ndarray:
    """Smooth random perturbation of a uniform state (rho, u, v, w, p) =
    (1, 0.3, -0.2, 0.1, 1/gamma) built from a few random Fourier modes per
    field, so RHS values are O(1) and every reconstruction branch is exercised."""
    mz, my, mx = shape
    rng = np.random.default_rng(seed)
    nn = (mx - 2, my - 2, mz - 2) if periodic else (mx, my, mz)
    k_ax = [2 * math.pi * (np.arange(m) - 1.0) / max(n, 1) for m, n in zip((mx, my, mz), nn)]
    z, y, x = np.meshgrid(k_ax[2], k_ax[1], k_ax[0], indexing="ij")
    base = [1.0, 0.3, -0.2, 0.1, 1.0 / gamma]
    fields = []
    for b in base:
        f = np.full(x.shape, b)
        for _ in range(4):
            kx, ky, kz = rng.integers(-3, 4, size=3)
            ph = rng.uniform(0, 2 * math.pi)
            a = rng.uniform(-amp, amp)
            f = f + a * np.cos(kx * x + ky * y + kz * z + ph)
        fields.append(f)
    rho, u, v, w, p = fields
    return conserved(rho, u, v, w, p, gamma)
