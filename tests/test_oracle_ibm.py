"""The oracle's restatement of the immersed-boundary interpolation
(ibm_interpolation_advanced, ibm_iso.c:2572-2880) and of immersed time steps
(solvers.c:282-288), pinned against the reference's own outputs: the golden
fixtures made by tests/golden/make_ibm_golden.py, and, where the reference
sources are present, the reference itself on synthetic lists."""
import numpy as np
import pytest

import oracle as O
from chimera_comp_les_b200 import _lib
from chimera_comp_les_b200 import workloads as W

from _common import ibm_golden_names, load_ibm_golden, synthetic_ibm_list

NAMES = ibm_golden_names()


def _oracle_interp(cfg, g, info, surf):
    o = O.Oracle(cfg)
    q = o.fill_ghosts(O.to_padded(cfg, g["q"]))
    p = o.eos(q)
    o.ibm_interpolate(O.IbmSurface(surf, g["u"], g["uold"]), info, O.to_padded(cfg, g["coords"]), q, p, 1)
    return O.from_padded(q), O.from_padded(p)[..., 0]


def test_fixtures_present():
    assert len(NAMES) >= 7


@pytest.mark.parametrize("name", NAMES)
def test_oracle_interpolation_bitwise_vs_reference(name):
    cfg, meta, g, info, surf = load_ibm_golden(name)
    q, p = _oracle_interp(cfg, g, info, surf)
    k, j, i = info["nk"], info["nj"], info["ni"]
    assert np.array_equal(q[k, j, i], g["q_interp"])
    assert np.array_equal(p[k, j, i], g["p_interp"])
    rest = np.ones(q.shape[:3], dtype=bool)
    rest[k, j, i] = False
    assert np.array_equal(q[rest], g["q"][rest])


@pytest.mark.parametrize("name", NAMES)
def test_oracle_immersed_steps_bitwise_vs_reference(name):
    cfg, meta, g, info, surf = load_ibm_golden(name)
    o = O.Oracle(cfg)
    if cfg.bctype[4] in (52, 47):  # the inflow codes read the node coordinates
        o.set_coordinates(O.to_padded(cfg, g["coords"]))
    met = o.metrics(o.fill_ghosts(O.to_padded(cfg, g["coords"])))
    nvp = o.fill_ghosts(O.to_padded(cfg, g["nvert"]))
    st = o.initial_state(g["q"])
    o.steps_immersed(meta["steps"], st, met, nvp, O.IbmSurface(surf, g["u"], g["uold"]), info,
                     O.to_padded(cfg, g["coords"]))
    assert np.array_equal(O.from_padded(st["q"]), g["q_steps"])


def test_list_layout_matches_the_c_struct():
    # cb_ibm_info / cbo_ibm_info: 14 ints then 11 doubles, 144 bytes
    assert O.IBM_INFO_DTYPE.itemsize == 144 and _lib.IBM_INFO_DTYPE.itemsize == 144
    assert O.IBM_INFO_DTYPE == _lib.IBM_INFO_DTYPE
    assert O.IBM_INFO_DTYPE.fields["cr1"][1] == 56


def test_flat_list_round_trip():
    cfg, meta, g, info, surf = load_ibm_golden(NAMES[0])
    iv, rv = O.ibm_info_to_flat(info)
    back = O.ibm_info_from_flat(iv, rv)
    assert np.array_equal(back, info)


def test_unsupported_variants_are_refused():
    cfg, meta, g, info, surf = load_ibm_golden(NAMES[0])
    # -wallfunction 1 reads a table left in a dead stack frame (wallfunction.c:113-145)
    for kw in (dict(wallfunction=1),):
        c2 = O.Config(**{**cfg.__dict__, **kw})
        with pytest.raises(RuntimeError):
            _oracle_interp(c2, g, info, surf)


def test_sphere_surface_is_closed_and_outward():
    s = W.sphere_surface(1.0, (0.5, -0.2, 0.1), 2)
    P = np.stack([s["x"], s["y"], s["z"]], 1)
    tri = np.stack([s["nv1"], s["nv2"], s["nv3"]], 1)
    # every edge is shared by exactly two triangles (a closed surface)
    edges = {}
    for t in tri:
        for a, b in ((t[0], t[1]), (t[1], t[2]), (t[2], t[0])):
            key = (min(a, b), max(a, b))
            edges[key] = edges.get(key, 0) + 1
    assert set(edges.values()) == {2}
    cen = P[tri].mean(axis=1) - np.array([0.5, -0.2, 0.1])
    nf = np.stack([s["nf_x"], s["nf_y"], s["nf_z"]], 1)
    assert np.all(np.einsum("ij,ij->i", cen, nf) > 0)
    assert np.allclose(np.linalg.norm(nf, axis=1), 1.0)


SYN_CASES = [
    ("noslip_iso1", dict(inviscid=0, isothermal=1)),
    ("freeslip_iso0", dict(inviscid=1, isothermal=0)),
    ("wf3_twoD3_iso1", dict(inviscid=0, isothermal=1, wallfunction=3, twoD=3)),
    # the hydset log law of the wall (wallfunction.c:376-420), which takes
    # precedence over freeslip with -inv (ibm_iso.c:2708-2728)
    # (Re 30000 puts the donor points at y+ from 11.53 to beyond 300: the
    # viscous sublayer, the log law and the reference's y+ > 300 fallback)
    ("wf2_loglaw", dict(inviscid=0, isothermal=0, wallfunction=2, ren=30000.)),
    ("wf2_sublayer_inv_iso1_twoD2", dict(inviscid=1, isothermal=1, wallfunction=2, twoD=2)),
    # the characteristic isothermal wall (ibm_iso.c:2744-2786): the scalar Pa
    # links each entry to the one walked before it, duplicates included
    ("iso2_noslip", dict(inviscid=0, isothermal=2)),
    ("iso2_twall_wf2_twoD1", dict(inviscid=0, isothermal=2, twall=1.3, wallfunction=2, twoD=1, ren=3000.)),
]


@pytest.mark.skipif(not O.ref_available(), reason="reference sources not present")
@pytest.mark.parametrize("name,kw", SYN_CASES, ids=[c[0] for c in SYN_CASES])
def test_oracle_interpolation_bitwise_vs_reference_synthetic_list(name, kw):
    """Duplicate nodes, donor chains and the element-normal fallback, on a
    non-uniform grid: the restatement against ibm_interpolation_advanced."""
    n = (19, 17, 18)
    coords = W.periodic_grid(n, 2 * np.pi, amp=0.05)
    shape = coords.shape[:3]
    cfg = O.Config(**{**dict(mx=n[0] + 2, my=n[1] + 2, mz=n[2] + 2, les=0, fluxorder=3, ren=300., ma=0.3, pr=0.71,
                             dt=0.002), **kw})
    surf = W.sphere_surface(2.0, coords[shape[0] // 2, shape[1] // 2, shape[2] // 2], 2)
    info = synthetic_ibm_list(cfg, coords, len(surf["nv1"]), seed=7)
    rng = np.random.default_rng(8)
    u = rng.normal(size=(len(surf["x"]), 3)) * 0.1
    uold = u * 0.9
    q = W.random_smooth_state(shape, seed=12)
    ref = O.RefOracle(cfg, coords)
    ref.ibm_setup(surf)
    ref.ibm_set_list(info)
    ref.ibm_set_velocity(u, uold)
    ref.set_state(q)
    ref.ibm_interpolate(1)
    o = O.Oracle(cfg)
    qp = o.fill_ghosts(O.to_padded(cfg, q))
    p = o.eos(qp)
    o.ibm_interpolate(O.IbmSurface(surf, u, uold), info, O.to_padded(cfg, coords), qp, p, 1)
    assert np.array_equal(O.from_padded(qp), ref.Q())
    assert np.array_equal(O.from_padded(p)[..., 0], ref.P())
