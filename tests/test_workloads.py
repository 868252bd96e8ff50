"""Host-side logic: synthetic workloads and layout helpers."""
import math

import numpy as np

import oracle as O
from chimera_comp_les_b200 import workloads as W


def test_periodic_grid_images():
    c = W.periodic_grid(8, 2 * math.pi)
    assert c.shape == (10, 10, 10, 3)
    dx = 2 * math.pi / 8
    assert np.allclose(c[0, 0, :, 0], (np.arange(10) - 1) * dx)
    # node m-1 is one period beyond node 1, node 0 one period before node m-2
    assert np.allclose(c[:, :, -1, 0] - c[:, :, 1, 0], 2 * math.pi)
    assert np.allclose(c[:, :, -2, 0] - c[:, :, 0, 0], 2 * math.pi)


def test_perturbed_grid_is_periodic_in_displacement():
    c0 = W.periodic_grid(8, 2 * math.pi)
    c1 = W.periodic_grid(8, 2 * math.pi, amp=0.05)
    d = c1 - c0
    assert np.allclose(d[:, :, 0], d[:, :, -2]) and np.allclose(d[:, :, 1], d[:, :, -1])
    assert np.abs(d).max() > 0.01


def test_tgv_state_reference_scaling():
    c = W.periodic_grid(8, 2 * math.pi)
    q = W.tgv_state(c, gamma=1.4, ma=0.1)
    x, y, z = c[..., 0], c[..., 1], c[..., 2]
    p = 100 + (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2) / 16
    assert np.allclose(q[..., 0], 1.4 * p * 0.01)
    assert np.allclose(q[..., 1], np.sin(x) * np.cos(y) * np.cos(z))


def test_vortex_free_stream_far_away():
    c = W.periodic_grid(16, 10.0)
    q = W.vortex_state(c)
    # Shu vortex with beta = 5: rho_min = (1 - 0.4*25*e/(8*1.4*pi^2))^2.5 = 0.494
    assert abs(q[0, 0, 0, 0] - 1.0) < 1e-3 and abs(q[..., 0].min() - 0.4938) < 2e-3


def test_padded_roundtrip():
    cfg = O.Config(mx=7, my=8, mz=9)
    a = np.random.default_rng(0).standard_normal((9, 8, 7, 5))
    assert np.array_equal(O.from_padded(O.to_padded(cfg, a)), a)


def test_clustered_axis_spacing():
    x = W.clustered_axis(192, -6.0, 6.0, 0.01)
    dx = np.diff(x)
    assert x[0] == -6.0 and x[-1] == 6.0 and np.all(dx > 0)
    assert abs(dx.min() - 0.01) < 1e-4 and abs(x[np.argmin(dx)]) < 0.02
    z = W.clustered_axis(256, -5.0, 15.0, 0.01)
    assert abs(np.diff(z).min() - 0.01) < 1e-4 and abs(z[np.argmin(np.diff(z))]) < 0.02


def test_sphere_case_list_is_consistent():
    n = (40, 36, 48)
    c = W.sphere_case(n=n, h_min=0.05)
    nv, info, coords = c["nvert"], c["info"], c["coords"]
    assert nv.shape == (48, 36, 40)
    k, j, i = info["nk"], info["nj"], info["ni"]
    assert np.all(nv[k, j, i] == 1.0) and info.size == int((nv == 1.0).sum())
    assert len(set(zip(i, j, k))) == info.size
    r = np.linalg.norm(coords[nv == 3.0], axis=1)
    assert np.all(r < 0.5)
    assert np.allclose(np.linalg.norm(info["pmin"], axis=1), 0.5)
    w = np.stack([info["cr1"], info["cr2"], info["cr3"]], 1)
    assert np.all(w > 0) and np.allclose(w.sum(1), 1.0)
    for a, b, cc in (("i1", "j1", "k1"), ("i2", "j2", "k2"), ("i3", "j3", "k3")):
        assert np.all(np.abs(info[a] - i) <= 2) and np.all(np.abs(info[b] - j) <= 2) and np.all(np.abs(info[cc] - k) <= 2)
        assert np.all(nv[info[cc], info[b], info[a]] == 0.0)
    assert np.all(info["d_s"] > 0) and np.all(info["d_i"] > 0)
    assert info["cell"].min() >= 0 and info["cell"].max() < len(c["surface"]["nv1"])
