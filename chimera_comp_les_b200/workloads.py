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


def periodic_grid_slab(n, length, amp: float, k0: int, mz: int) -> np.ndarray:
    """Nodes k0 .. k0+mz-1 (global DMDA k index) of ``periodic_grid(n, length,
    amp)``, without building the whole box."""
    ns = tuple(n)
    ls = tuple(length)
    ax = [(np.arange(ns[d] + 2) - 1.0) * (ls[d] / ns[d]) for d in range(3)]
    z, y, x = np.meshgrid(ax[2][k0:k0 + mz], ax[1], ax[0], indexing="ij")
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


def distorted_periodic_grid(n, length, amp: float, seed: int, modes: int = 3) -> np.ndarray:
    """Periodic box (n, length as in ``periodic_grid``) whose nodes are moved
    by a seeded smooth random field: every coordinate gets a sum of `modes`
    periodic sine modes (wavenumbers 1..2 per direction, random phases) scaled
    so the largest displacement is `amp`."""
    ns = (n, n, n) if np.isscalar(n) else tuple(int(x) for x in n)
    ls = (length, length, length) if np.isscalar(length) else tuple(length)
    g = periodic_grid(ns, ls, 0.0)
    rng = np.random.default_rng(seed)
    xi = [2 * math.pi * (np.arange(ns[d] + 2) - 1.0) / ns[d] for d in range(3)]
    z, y, x = np.meshgrid(xi[2], xi[1], xi[0], indexing="ij")
    out = g.copy()
    for c in range(3):
        f = np.zeros_like(x)
        for _ in range(modes):
            kx, ky, kz = rng.integers(0, 3, size=3)
            if kx == ky == kz == 0:
                kx = 1
            f += rng.uniform(-1, 1) * np.sin(kx * x + ky * y + kz * z + rng.uniform(0, 2 * math.pi))
        m = np.abs(f).max()
        if m > 0:
            out[..., c] += amp * f / m
    return np.ascontiguousarray(out)


def _spectrum(kind: str, k: np.ndarray, k_peak: float) -> np.ndarray:
    if kind == "von_karman":  # E ~ (k/kp)^4 / (1 + (k/kp)^2)^(17/6)
        r = k / k_peak
        return r ** 4 / (1.0 + r * r) ** (17.0 / 6.0)
    if kind == "passot_pouquet":  # E ~ (k/k0)^4 exp(-2 (k/k0)^2)
        r = k / k_peak
        return r ** 4 * np.exp(-2.0 * r * r)
    raise ValueError(kind)


def isotropic_turbulence(n, seed: int, k_peak: float = 4.0, mach_t: float = 0.3, spectrum: str = "von_karman",
                         gamma: float = 1.4, u_rms: float | None = None) -> np.ndarray:
    """Solenoidal random velocity field with energy spectrum `spectrum` peaking
    near k_peak (integer wavenumbers of a 2*pi box) and random phases from
    `seed`, on rho = 1 and a uniform pressure.  Without u_rms: sound speed 1
    (p = 1/gamma) and the field scaled so sqrt(<u.u>) = mach_t.  With u_rms:
    each component has that rms and p is set so sqrt(<u.u>) / c = mach_t.
    n: unique points (nx, ny, nz); returns the state on the DMDA nodes
    (nz+2, ny+2, nx+2, 5) with the periodic images."""
    nx, ny, nz = (n, n, n) if np.isscalar(n) else tuple(int(x) for x in n)
    rng = np.random.default_rng(seed)
    kx, ky, kz = (np.fft.fftfreq(m, 1.0 / m) for m in (nx, ny, nz))
    KZ, KY, KX = np.meshgrid(kz, ky, kx, indexing="ij")
    k2 = KX * KX + KY * KY + KZ * KZ
    k = np.sqrt(k2)
    amp = np.zeros_like(k)
    # no Nyquist modes (their -k is the same coefficient, which breaks the projection)
    nz_ = (k > 0) & (2 * np.abs(KX) < nx) & (2 * np.abs(KY) < ny) & (2 * np.abs(KZ) < nz)
    amp[nz_] = np.sqrt(_spectrum(spectrum, k[nz_], k_peak) / (4 * math.pi * k2[nz_]))
    uh = [amp * (rng.standard_normal(k.shape) + 1j * rng.standard_normal(k.shape)) for _ in range(3)]
    kdu = KX * uh[0] + KY * uh[1] + KZ * uh[2]
    inv = np.zeros_like(k)
    inv[nz_] = 1.0 / k2[nz_]
    uh = [uh[0] - KX * kdu * inv, uh[1] - KY * kdu * inv, uh[2] - KZ * kdu * inv]
    u = [np.real(np.fft.ifftn(a)) for a in uh]
    if u_rms is not None:
        s = u_rms / math.sqrt(np.mean((u[0] ** 2 + u[1] ** 2 + u[2] ** 2) / 3.0))
    else:
        s = mach_t / math.sqrt(np.mean(u[0] ** 2 + u[1] ** 2 + u[2] ** 2))
    u = [a * s for a in u]
    c = math.sqrt(np.mean(u[0] ** 2 + u[1] ** 2 + u[2] ** 2)) / mach_t if u_rms is not None else 1.0
    iz, iy, ix = ((np.arange(m + 2) - 1) % m for m in (nz, ny, nx))
    u = [a[np.ix_(iz, iy, ix)] for a in u]
    rho = np.ones_like(u[0])
    p = np.full_like(u[0], c * c / gamma)
    return conserved(rho, u[0], u[1], u[2], p, gamma)


def multiblock_set(seed: int = 2024, nblocks: int = 24, ranges=((32, 160), (32, 128), (32, 96)), amp: float = 0.03,
                   k_peak: float = 4.0, mach_t: float = 0.3, gamma: float = 1.4, cfl: float = 0.4):
    """Uneven multi-block set: block sizes (unique points per direction) drawn
    uniformly from `ranges`, each block a [0, 2*pi]^3 box with a seeded smooth
    metric distortion of amplitude `amp` carrying decaying isotropic turbulence
    (von Karman spectrum, k_peak, turbulent Mach mach_t), and a seeded donor
    permutation without fixed points for the 2-node overlap halo.

    Returns dict(dims=[(mx, my, mz)] DMDA node counts, coords=[...], q=[...],
    perm=[...], dt=...) with dt from the CFL estimate
    cfl / max_b sum_d (max|u| + c) * N_d / (2*pi) * 1.2."""
    rng = np.random.default_rng(seed)
    uniq = [tuple(int(rng.integers(lo, hi + 1)) for lo, hi in ranges) for _ in range(nblocks)]
    while True:
        perm = rng.permutation(nblocks)
        if nblocks == 1 or not (perm == np.arange(nblocks)).any():
            break
    coords, qs = [], []
    lam = 0.0
    for b, n in enumerate(uniq):
        coords.append(distorted_periodic_grid(n, 2 * math.pi, amp, seed=seed * 1000 + 2 * b))
        q = isotropic_turbulence(n, seed * 1000 + 2 * b + 1, k_peak=k_peak, mach_t=mach_t, gamma=gamma)
        qs.append(q)
        umax = float(np.abs(q[..., 1:4] / q[..., :1]).max())
        lam = max(lam, sum((umax + 1.0) * n[d] / (2 * math.pi) for d in range(3)) * 1.2)
    dt = math.floor(cfl / lam * 1e5) / 1e5
    return dict(dims=[(n[0] + 2, n[1] + 2, n[2] + 2) for n in uniq], coords=coords, q=qs,
                perm=[int(x) for x in perm], dt=dt)


def sphere_surface(radius: float, center=(0.0, 0.0, 0.0), subdiv: int = 3):
    """Triangulated sphere (a subdivided icosahedron projected onto the
    sphere), in the arrays of the reference's IBM surface (IBMNodes,
    variables.h:91-118): vertex coordinates x, y, z (n_v each), triangles
    nv1, nv2, nv3 (n_elmt each, counter-clockwise seen from outside), and the
    unit normals nf_x, nf_y, nf_z of each triangle, (p2 - p1) x (p3 - p1)
    normalised, pointing out of the body (ibm_read_ucd
    forms them the same way, ibm_io.c:1718-1732)."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
             (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    v = [np.array(p, dtype=np.float64) / np.linalg.norm(p) for p in verts]
    for _ in range(subdiv):
        mid = {}

        def midpoint(a, b):
            key = (min(a, b), max(a, b))
            if key not in mid:
                m = v[a] + v[b]
                v.append(m / np.linalg.norm(m))
                mid[key] = len(v) - 1
            return mid[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = midpoint(a, b), midpoint(b, c), midpoint(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    P = np.array(v) * radius + np.asarray(center, dtype=np.float64)
    tri = np.array(faces, dtype=np.int32)
    d12 = P[tri[:, 1]] - P[tri[:, 0]]
    d13 = P[tri[:, 2]] - P[tri[:, 0]]
    n = np.cross(d12, d13)
    n /= np.linalg.norm(n, axis=1)[:, None]
    return {"x": P[:, 0].copy(), "y": P[:, 1].copy(), "z": P[:, 2].copy(),
            "nv1": tri[:, 0].copy(), "nv2": tri[:, 1].copy(), "nv3": tri[:, 2].copy(),
            "nf_x": n[:, 0].copy(), "nf_y": n[:, 1].copy(), "nf_z": n[:, 2].copy()}


# ------------------------------------------------------------ sphere flow --
def clustered_axis(n: int, a: float, b: float, h_min: float, x0: float = 0.0) -> np.ndarray:
    """n node positions on [a, b] clustered at x0 by a hyperbolic-sine map,
    x(s) = x0 + A sinh(beta (s - s0)), s uniform on [0, 1], with the spacing at
    x0 equal to h_min (A beta = h_min (n - 1))."""
    if not (a < x0 < b) or h_min * (n - 1) >= (b - a):
        raise ValueError("clustered_axis: x0 must lie inside (a, b) and h_min be below the uniform spacing")
    ga = h_min * (n - 1)

    def s0_for(beta):  # x(0) = a, x(1) = b fix s0 for a given beta
        lo, hi = 0.0, 1.0
        for _ in range(200):
            s0 = 0.5 * (lo + hi)
            r = math.sinh(beta * (1 - s0)) / math.sinh(beta * s0)
            if r > (b - x0) / (x0 - a):
                lo = s0
            else:
                hi = s0
        return 0.5 * (lo + hi)

    def span(beta):  # b - a produced by (beta, s0(beta)) at the given centre spacing
        s0 = s0_for(beta)
        A = ga / beta
        return A * (math.sinh(beta * (1 - s0)) + math.sinh(beta * s0)), s0

    lo, hi = 1e-6, 60.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if span(mid)[0] < (b - a):
            lo = mid
        else:
            hi = mid
    beta = 0.5 * (lo + hi)
    s0 = s0_for(beta)
    s = np.arange(n) / (n - 1.0)
    x = x0 + (ga / beta) * np.sinh(beta * (s - s0))
    x[0], x[-1] = a, b
    return x


def sphere_case(n=(192, 192, 256), diameter: float = 1.0, h_min: float = 0.01, ma: float = 0.3,
                gamma: float = 1.4, noise: float = 1e-3, seed: int = 3, subdiv: int = 4):
    """Flow past a stationary sphere: streamwise k on [-5, 15] D, i and j on
    [-6, 6] D, nodes clustered toward the sphere at the origin (spacing h_min D
    there); n = DMDA node counts (mx, my, mz).  The sphere marks nvert in the
    reference's encoding (ibm_iso.c:765-766): 3 inside, 1 on interface nodes
    (outside, with an inside node among their 26 neighbours), 0 in the fluid.
    State: uniform stream rho = 1, w = 1, p = 1/(gamma Ma^2) (the inflow of
    bctype 45, rhs.c:889-892) plus seeded white noise of amplitude `noise` on
    the three velocity components.  Returns coords, q, nvert, the surface
    (sphere_surface) and the interpolation list (sphere_ibm_list)."""
    mx, my, mz = n
    D = diameter
    xs = clustered_axis(mx, -6 * D, 6 * D, h_min * D)
    ys = clustered_axis(my, -6 * D, 6 * D, h_min * D)
    zs = clustered_axis(mz, -5 * D, 15 * D, h_min * D)
    z, y, x = np.meshgrid(zs, ys, xs, indexing="ij")
    coords = np.ascontiguousarray(np.stack([x, y, z], axis=-1))
    r = np.sqrt(x * x + y * y + z * z)
    inside = r < 0.5 * D
    near = np.zeros_like(inside)
    ii = np.argwhere(inside)
    for dk in (-1, 0, 1):
        for dj in (-1, 0, 1):
            for di in (-1, 0, 1):
                k = np.clip(ii[:, 0] + dk, 0, mz - 1)
                j = np.clip(ii[:, 1] + dj, 0, my - 1)
                i = np.clip(ii[:, 2] + di, 0, mx - 1)
                near[k, j, i] = True
    nvert = np.zeros((mz, my, mx))
    nvert[near & ~inside] = 1.0
    nvert[inside] = 3.0
    rng = np.random.default_rng(seed)
    u = noise * rng.standard_normal((mz, my, mx))
    v = noise * rng.standard_normal((mz, my, mx))
    w = 1.0 + noise * rng.standard_normal((mz, my, mx))
    rho = np.ones((mz, my, mx))
    p = np.full((mz, my, mx), 1.0 / (gamma * ma * ma))
    q = conserved(rho, u, v, w, p, gamma)
    surf = sphere_surface(0.5 * D, (0.0, 0.0, 0.0), subdiv)
    info = sphere_ibm_list(coords, nvert, (0.0, 0.0, 0.0), 0.5 * D, surf)
    return {"coords": coords, "q": q, "nvert": nvert, "surface": surf, "info": info,
            "bctype": (3, 3, 3, 3, 45, 45)}


IBM_LIST_FIELDS = [
    ("ni", "<i4"), ("nj", "<i4"), ("nk", "<i4"), ("cell", "<i4"),
    ("i1", "<i4"), ("j1", "<i4"), ("k1", "<i4"), ("i2", "<i4"), ("j2", "<i4"), ("k2", "<i4"),
    ("i3", "<i4"), ("j3", "<i4"), ("k3", "<i4"), ("pad", "<i4"),
    ("cr1", "<f8"), ("cr2", "<f8"), ("cr3", "<f8"), ("cs1", "<f8"), ("cs2", "<f8"), ("cs3", "<f8"),
    ("d_s", "<f8"), ("d_i", "<f8"), ("pmin", "<f8", (3,)),
]


def sphere_ibm_list(coords: np.ndarray, nvert: np.ndarray, center, radius: float, surf: dict) -> np.ndarray:
    """An interpolation list for an analytic sphere, in the entry layout of
    cb_ibm_info.  A stand-in for the reference's ray-casting search
    (ibm_search_advanced, which stays on the host): for every interface node
    (nvert 1) the interception point pmin is the nearest point of the sphere,
    d_s the distance to it, the donor point lies one local grid spacing d_i
    further out along the normal, and its three nearest fluid nodes (nvert 0)
    within two nodes carry inverse-distance weights.  The surface element is
    the triangle whose centroid is nearest to pmin, with equal vertex weights."""
    c = np.asarray(center, dtype=np.float64)
    nodes = np.argwhere(nvert == 1.0)  # (k, j, i)
    mz, my, mx = nvert.shape
    X = coords[nodes[:, 0], nodes[:, 1], nodes[:, 2]]
    d = X - c
    r = np.linalg.norm(d, axis=1)
    nrm = d / r[:, None]
    pmin = c + radius * nrm
    d_s = r - radius
    # local spacing: the shortest edge to a neighbour along i, j, k
    h = np.full(len(nodes), np.inf)
    for ax, lim in ((2, mx), (1, my), (0, mz)):
        for s in (-1, 1):
            nb = nodes.copy()
            nb[:, ax] = np.clip(nb[:, ax] + s, 0, lim - 1)
            e = np.linalg.norm(coords[nb[:, 0], nb[:, 1], nb[:, 2]] - X, axis=1)
            h = np.minimum(h, np.where(e > 0, e, np.inf))
    xd = X + nrm * h[:, None]
    offs = np.array([(a, b, cc) for a in range(-2, 3) for b in range(-2, 3) for cc in range(-2, 3)])
    cand = nodes[:, None, :] + offs[None, :, :]
    lim = np.array([mz, my, mx])
    valid = np.all((cand >= 0) & (cand < lim), axis=2)
    cc_ = np.clip(cand, 0, lim - 1)
    fluid = valid & (nvert[cc_[..., 0], cc_[..., 1], cc_[..., 2]] == 0.0)
    dist = np.linalg.norm(coords[cc_[..., 0], cc_[..., 1], cc_[..., 2]] - xd[:, None, :], axis=2)
    dist = np.where(fluid, dist, np.inf)
    pick = np.argsort(dist, axis=1)[:, :3]
    dd = np.take_along_axis(dist, pick, axis=1)
    if not np.all(np.isfinite(dd)):
        raise ValueError("sphere_ibm_list: an interface node has fewer than three fluid nodes within two nodes")
    wgt = 1.0 / np.maximum(dd, 1e-12)
    wgt /= wgt.sum(axis=1, keepdims=True)
    don = np.take_along_axis(cand, pick[:, :, None], axis=1)  # (n, 3, (k, j, i))
    # nearest surface element by centroid, in chunks
    P = np.stack([surf["x"], surf["y"], surf["z"]], 1)
    cen = (P[surf["nv1"]] + P[surf["nv2"]] + P[surf["nv3"]]) / 3.0
    cell = np.empty(len(nodes), dtype=np.int32)
    for a in range(0, len(nodes), 4096):
        dc = np.linalg.norm(pmin[a:a + 4096, None, :] - cen[None, :, :], axis=2)
        cell[a:a + 4096] = np.argmin(dc, axis=1)
    out = np.zeros(len(nodes), dtype=np.dtype(IBM_LIST_FIELDS))
    out["nk"], out["nj"], out["ni"] = nodes[:, 0], nodes[:, 1], nodes[:, 2]
    out["cell"] = cell
    for t, (a, b, cc) in enumerate((("i1", "j1", "k1"), ("i2", "j2", "k2"), ("i3", "j3", "k3"))):
        out[cc], out[b], out[a] = don[:, t, 0], don[:, t, 1], don[:, t, 2]
    out["cr1"], out["cr2"], out["cr3"] = wgt[:, 0], wgt[:, 1], wgt[:, 2]
    out["cs1"] = out["cs2"] = out["cs3"] = 1.0 / 3.0
    out["d_s"], out["d_i"] = d_s, h
    out["pmin"] = pmin
    return out
