"""GPU parity of the immersed-boundary path (cb_ibm_*): the interpolation
(ibm_interpolation_advanced, ibm_iso.c:2572-2880) and immersed time steps
(RungeKutta with -imm, solvers.c:245-288) against the reference's outputs
(tests/golden/ibm, made by the reference's own search and interpolation) and
against the oracle restatement.

Bar (FP64 form): per conserved field, relative L2 <= 1e-12 (RTOL_L2)."""
import numpy as np
import pytest

import oracle as O
from chimera_comp_les_b200 import ChimeraError
from chimera_comp_les_b200 import workloads as W

from _common import (RTOL_L2, gpu_block, gpu_ibm_block, ibm_golden_names, load_ibm_golden, per_field_rel_l2,
                     synthetic_ibm_list)

pytestmark = pytest.mark.gpu

NAMES = ibm_golden_names()


def _fixture_block(name, precision="fp64"):
    cfg, meta, g, info, surf = load_ibm_golden(name)
    b = gpu_ibm_block(cfg, g["coords"], g["nvert"], g["q"], surf, info, g["u"], g["uold"], precision)
    return cfg, meta, g, info, b


@pytest.mark.parametrize("name", NAMES)
def test_interpolation_matches_reference(name):
    cfg, meta, g, info, b = _fixture_block(name)
    with b:
        assert b.ibm_count(0) == info.size
        b.ibm_interpolation_advanced(0, 1)
        q = b.Q()
        p = b.EqOfState()
    k, j, i = info["nk"], info["nj"], info["ni"]
    assert max(per_field_rel_l2(q[k, j, i], g["q_interp"])) <= RTOL_L2
    assert O.rel_l2(p[k, j, i], g["p_interp"]) <= RTOL_L2
    rest = np.ones(q.shape[:3], dtype=bool)
    rest[k, j, i] = False
    assert np.array_equal(q[rest], g["q"][rest])


@pytest.mark.parametrize("name", NAMES)
def test_immersed_steps_match_reference(name):
    cfg, meta, g, info, b = _fixture_block(name)
    with b:
        b.RungeKutta(meta["steps"])
        q = b.Q()
    errs = per_field_rel_l2(q, g["q_steps"])
    assert max(errs) <= RTOL_L2, errs


def _synthetic_case(seed=5, n=(37, 29, 33), **kw):
    coords = W.periodic_grid(n, 2 * np.pi, amp=0.04)
    shape = coords.shape[:3]
    base = dict(les=1, inviscid=0, fluxorder=3, ren=500., ma=0.3, pr=0.71, dt=0.002, isothermal=1)
    base.update(kw)
    cfg = O.Config(mx=n[0] + 2, my=n[1] + 2, mz=n[2] + 2, immersed=1, **base)
    surf = W.sphere_surface(2.0, coords[shape[0] // 2, shape[1] // 2, shape[2] // 2], 2)
    info = synthetic_ibm_list(cfg, coords, len(surf["nv1"]), seed=seed, radius=6.0)
    rng = np.random.default_rng(seed)
    u = rng.normal(size=(len(surf["x"]), 3)) * 0.02
    uold = u * 0.99
    q = W.random_smooth_state(shape, seed=seed)
    nv = np.zeros(shape)
    nv[info["nk"], info["nj"], info["ni"]] = 1.0
    return cfg, coords, q, nv, surf, info, u, uold


SYN = [
    ("les_noslip_periodic", {}),
    ("inviscid_iso0_kflow", dict(les=0, inviscid=1, isothermal=0, bctype=(7, 7, 7, 7, 45, 45))),
    ("visc_wf3_walls", dict(les=0, wallfunction=3, bctype=(7, 7, 3, 3, 44, 44))),
    # the hydset log law of -wallfunction 2 (wallfunction.c:376-420): at Re
    # 30000 the donor points sit in the log layer and beyond y+ = 300
    ("les_wf2_loglaw", dict(wallfunction=2, ren=30000.)),
    ("visc_wf2_walls_iso0", dict(les=0, wallfunction=2, isothermal=0, ren=3000., bctype=(7, 7, 3, 3, 44, 44))),
    # the characteristic isothermal wall of -isothermal 2 (ibm_iso.c:2744-2786):
    # the pressure Pa chains every entry, duplicates included, to the one
    # walked before it; with the j walls of code 1 its FormBCS counterpart
    ("visc_iso2_walls44", dict(les=0, isothermal=2, twall=1.2, bctype=(7, 7, 3, 3, 44, 44))),
    ("les_iso2_jwalls1_wf2", dict(isothermal=2, twall=1.1, wallfunction=2, ren=3000., bctype=(7, 7, 1, 1, 7, 7))),
]


@pytest.mark.parametrize("name,kw", SYN, ids=[s[0] for s in SYN])
def test_synthetic_list_steps_match_oracle(name, kw):
    """Duplicate nodes (the later entry wins), donors that are interface nodes
    (sweeps chain), the element-normal fallback, a moving surface; several
    tiles and k-chunks."""
    cfg, coords, q, nv, surf, info, u, uold = _synthetic_case(**kw)
    o = O.Oracle(cfg)
    met = o.metrics(o.fill_ghosts(O.to_padded(cfg, coords)))
    st = o.initial_state(q)
    o.steps_immersed(3, st, met, o.fill_ghosts(O.to_padded(cfg, nv)), O.IbmSurface(surf, u, uold), info,
                     O.to_padded(cfg, coords))
    with gpu_ibm_block(cfg, coords, nv, q, surf, info, u, uold) as b:
        unique = len({(a, c, d) for a, c, d in zip(info["ni"], info["nj"], info["nk"])})
        assert b.ibm_count(0) == (info.size if cfg.isothermal == 2 else unique)
        assert unique < info.size  # the list has duplicates
        b.RungeKutta(3)
        qd = b.Q()
        pd = b.EqOfState()
    assert max(per_field_rel_l2(qd, O.from_padded(st["q"]))) <= RTOL_L2
    assert O.rel_l2(pd, O.from_padded(st["lp"])[..., 0]) <= RTOL_L2


def test_two_bodies_in_order():
    cfg, coords, q, nv, surf, info, u, uold = _synthetic_case(seed=9)
    half = info.size // 2
    lists = [info[:half], info[half:]]
    o = O.Oracle(cfg)
    met = o.metrics(o.fill_ghosts(O.to_padded(cfg, coords)))
    st = o.initial_state(q)
    surfs = [O.IbmSurface(surf, u, uold), O.IbmSurface(surf, -u, -uold)]
    o.steps_immersed(2, st, met, o.fill_ghosts(O.to_padded(cfg, nv)), surfs, lists, O.to_padded(cfg, coords))
    with gpu_block(cfg) as b:
        b.FormMetrics(coords)
        b.set_nvert(nv)
        b.SetInitialCondition(q)
        for ibi, (lst, sgn) in enumerate(zip(lists, (1, -1))):
            b.set_ibm_surface(ibi, surf)
            b.set_ibm_velocity(ibi, sgn * u, sgn * uold)
            b.set_ibm_list(ibi, lst, coords)
        b.RungeKutta(2)
        qd = b.Q()
    assert max(per_field_rel_l2(qd, O.from_padded(st["q"]))) <= RTOL_L2


def test_graph_replay_equals_eager_with_bodies():
    cfg, coords, q, nv, surf, info, u, uold = _synthetic_case(seed=3, n=(30, 22, 26))
    with gpu_ibm_block(cfg, coords, nv, q, surf, info, u, uold) as b:
        b.RungeKutta(5)
        qa = b.Q()
    with gpu_ibm_block(cfg, coords, nv, q, surf, info, u, uold) as b:
        b.timing(True)
        b.RungeKutta(5)
        qb = b.Q()
    assert np.array_equal(qa, qb)


def test_mixed_form_with_bodies_tracks_fp64():
    cfg, coords, q, nv, surf, info, u, uold = _synthetic_case(seed=4, n=(40, 32, 36))
    out = {}
    for prec in ("fp64", "mixed"):
        with gpu_ibm_block(cfg, coords, nv, q, surf, info, u, uold, precision=prec) as b:
            b.RungeKutta(20)
            out[prec] = b.Q()
    assert max(per_field_rel_l2(out["mixed"], out["fp64"])) <= 1e-5


def test_removing_the_list_restores_plain_steps():
    cfg, coords, q, nv, surf, info, u, uold = _synthetic_case(seed=6, n=(24, 20, 22))
    with gpu_block(cfg) as b:
        b.FormMetrics(coords)
        b.set_nvert(nv)
        b.SetInitialCondition(q)
        b.RungeKutta(2)
        want = b.Q()
    with gpu_ibm_block(cfg, coords, nv, q, surf, info, u, uold) as b:
        b.set_ibm_list(0, info[:0], coords)
        assert b.ibm_count(0) == 0
        b.RungeKutta(2)
        assert np.array_equal(b.Q(), want)


def test_invalid_lists_and_options_fail_loudly():
    cfg, coords, q, nv, surf, info, u, uold = _synthetic_case(seed=2, n=(20, 18, 16))
    with gpu_block(cfg) as b:
        b.FormMetrics(coords)
        b.SetInitialCondition(q)
        with pytest.raises(ChimeraError) as ei:
            b.set_ibm_list(0, info, coords)  # no surface yet
        assert ei.value.code == 3
        b.set_ibm_surface(0, surf)
        bad = info.copy()
        bad[3]["i2"] = cfg.mx + 5
        with pytest.raises(ChimeraError) as ei:
            b.set_ibm_list(0, bad, coords)
        assert ei.value.code == 1
        bad = info.copy()
        bad[0]["cell"] = len(surf["nv1"])
        with pytest.raises(ChimeraError):
            b.set_ibm_list(0, bad, coords)
        with pytest.raises(ChimeraError) as ei:  # -wallfunction 1: the reference's table is undefined
            b.set_ibm_options(0, 1)
        assert ei.value.code == 5
        with pytest.raises(ChimeraError) as ei:
            b.set_ibm_options(0, 4)
        assert ei.value.code == 1
        with pytest.raises(ChimeraError):
            b.set_ibm_surface(16, surf)  # body index out of range (CB_IBM_MAX_BODIES)


def test_sphere_workload_small_matches_oracle():
    """The sphere workload (clustered grid, slip walls, inflow/outflow 45,
    Roe flux, analytic interpolation list) at 40 x 36 x 48 nodes: three
    immersed steps against the oracle in both the FP64 and mixed forms."""
    n = (40, 36, 48)
    case = W.sphere_case(n=n, h_min=0.05)
    cfg = O.Config(mx=n[0], my=n[1], mz=n[2], bctype=case["bctype"], les=1, inviscid=0, fluxorder=3, ren=300.,
                   ma=0.3, pr=0.71, dt=1e-3, cs_const=0.1, isothermal=0, flux=1, immersed=1)
    o = O.Oracle(cfg)
    met = o.metrics(O.to_padded(cfg, case["coords"]))
    st = o.initial_state(case["q"])
    o.steps_immersed(3, st, met, o.fill_ghosts(O.to_padded(cfg, case["nvert"])), O.IbmSurface(case["surface"]),
                     case["info"], O.to_padded(cfg, case["coords"]))
    want = O.from_padded(st["q"])
    for prec, tol in (("fp64", RTOL_L2), ("mixed", 1e-5)):
        with gpu_ibm_block(cfg, case["coords"], case["nvert"], case["q"], case["surface"], case["info"],
                           precision=prec) as b:
            b.RungeKutta(3)
            errs = per_field_rel_l2(b.Q(), want)
        assert max(errs) <= tol, (prec, errs)


def test_wall_function_ustar_matches_oracle():
    """-wallfunction 2: one interpolation (five sweeps); the state and u_tau of
    every kept entry (cb_ibm_get_ustar: the last entry of a node listed
    twice) against the restatement, which is bit-exact against the
    reference (tests/test_oracle_ibm.py).  The device's log / exp may differ
    from the host's in the last bit, so the bar is relative L2."""
    cfg, coords, q, nv, surf, info, u, uold = _synthetic_case(seed=6, wallfunction=2, ren=30000.)
    o = O.Oracle(cfg)
    qp = o.fill_ghosts(O.to_padded(cfg, q))
    p = o.eos(qp)
    us = np.zeros(info.size)
    o.ibm_interpolate(O.IbmSurface(surf, u, uold), info, O.to_padded(cfg, coords), qp, p, 1, ustar=us)
    last = {}
    for t, nd in enumerate(zip(info["ni"], info["nj"], info["nk"])):
        last[nd] = t
    keep = [t for t, nd in enumerate(zip(info["ni"], info["nj"], info["nk"])) if last[nd] == t]
    with gpu_ibm_block(cfg, coords, nv, q, surf, info, u, uold) as b:
        assert np.all(b.ibm_ustar(0) == 0)
        b.ibm_interpolation_advanced(0, 1)
        qd = b.Q()
        usd = b.ibm_ustar(0)
    assert usd.shape == (len(keep),) and np.all(usd > 0)
    assert O.rel_l2(usd, us[keep]) <= RTOL_L2
    assert max(per_field_rel_l2(qd, O.from_padded(qp))) <= RTOL_L2


def test_iso2_interpolation_matches_oracle():
    """-isothermal 2 alone (five sweeps, the chained Pa over a list with
    duplicates and donor chains) against the restatement, which is bit-exact
    against the reference (tests/test_oracle_ibm.py)."""
    cfg, coords, q, nv, surf, info, u, uold = _synthetic_case(seed=11, isothermal=2, twall=1.15, les=0)
    o = O.Oracle(cfg)
    qp = o.fill_ghosts(O.to_padded(cfg, q))
    p = o.eos(qp)
    o.ibm_interpolate(O.IbmSurface(surf, u, uold), info, O.to_padded(cfg, coords), qp, p, 1)
    with gpu_ibm_block(cfg, coords, nv, q, surf, info, u, uold) as b:
        b.ibm_interpolation_advanced(0, 1)
        qd = b.Q()
        pd = b.EqOfState()
    assert max(per_field_rel_l2(qd, O.from_padded(qp))) <= RTOL_L2
    k, j, i = info["nk"], info["nj"], info["ni"]
    assert O.rel_l2(pd[k, j, i], O.from_padded(p)[..., 0][k, j, i]) <= RTOL_L2
