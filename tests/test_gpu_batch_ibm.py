"""Immersed bodies in the batched form (cb_batch_ibm_*).

After the stages of a step the reference interpolates every body on every
block (ibm_interpolation_advanced with the block's list), then runs
FormBCS(user, 0) on it (solvers.c:279-288).  A batched block with face codes
and a body's list must advance exactly as a single-block context with the
same list (FP64 bit for bit, the mixed form within 1e-7 of its own
single-block run), next to an interface block of the halo maps; on the
reference-generated fixtures it must also match the reference's own steps
(relative L2 <= 1e-12, tests/golden/ibm).
"""
import numpy as np
import pytest

import oracle as O
from _common import RTOL_L2, gpu_ibm_block, load_ibm_golden, per_field_rel_l2, synthetic_ibm_list
from chimera_comp_les_b200 import workloads as W

pytestmark = pytest.mark.gpu

# the fixtures whose block has a physical face code (k-flow 45/45, walls 3 and 44)
CODED = ["sphere_kflow45", "sphere_les_walls44"]
IFACE = (20, 18, 16)  # the interface block beside the immersed one


def _batch_kwargs(cfg):
    return dict(les=cfg.les, inviscid=cfg.inviscid, fluxorder=cfg.fluxorder, eno_order=cfg.eno_order,
                central=cfg.central, isothermal=cfg.isothermal, s_x=cfg.s_x, s_y=cfg.s_y, s_z=cfg.s_z, ren=cfg.ren,
                ma=cfg.ma, pr=cfg.pr, gamma=cfg.gamma, dt=cfg.dt, st=cfg.st, cs_const=cfg.cs_const, ci=cfg.ci,
                ratio=cfg.ratio, calc_sigma=cfg.calc_sigma, s_x_min=cfg.s_x_min, s_y_min=cfg.s_y_min,
                s_z_min=cfg.s_z_min, sigma_thrsh=cfg.sigma_thrsh, flux=cfg.flux, twod=cfg.twoD, visT=cfg.visT,
                tref=cfg.tref, abc=cfg.abc, weno_order=cfg.weno_order, max_cs=cfg.max_cs, twall=cfg.twall)


def _iface_inputs():
    n = (IFACE[0] - 2, IFACE[1] - 2, IFACE[2] - 2)
    coords = W.periodic_grid(n, 2 * np.pi, amp=0.04)
    return coords, W.random_smooth_state(coords.shape[:3], seed=31, periodic=True)


def _run_batch(cfg, coords, nvert, q, surf, info, u, uold, steps, precision="fp64"):
    from chimera_comp_les_b200.batch import Batch
    dims = [(cfg.mx, cfg.my, cfg.mz), IFACE]
    ic, iq = _iface_inputs()
    with Batch(dims, precision=precision, **_batch_kwargs(cfg)) as bt:
        bt.set_bctype(0, tuple(cfg.bctype))
        bt.FormMetrics(0, coords)
        bt.set_nvert(0, nvert)
        bt.SetInitialCondition(0, q)
        bt.FormMetrics(1, ic)
        bt.SetInitialCondition(1, iq)
        bt.set_ibm_options(twoD=cfg.twoD, wallfunction=cfg.wallfunction)
        bt.set_ibm_surface(0, surf)
        if u is not None:
            bt.set_ibm_velocity(0, u, uold)
        bt.set_ibm_list(0, 0, info, coords)
        bt.halo_periodic()
        bt.RungeKutta(steps)
        return bt.Q(0), bt.Q(1)


def _single_iface(cfg, steps, precision):
    from chimera_comp_les_b200 import Block
    ic, iq = _iface_inputs()
    with Block(*IFACE, precision=precision, **_batch_kwargs(cfg)) as blk:
        blk.FormMetrics(ic)
        blk.SetInitialCondition(iq)
        blk.RungeKutta(steps)
        return blk.Q()


@pytest.mark.parametrize("name", CODED)
def test_immersed_block_matches_reference_and_single_block(name):
    cfg, meta, g, info, surf = load_ibm_golden(name)
    steps = meta["steps"]
    for prec in ("fp64", "mixed"):
        got, got_if = _run_batch(cfg, g["coords"], g["nvert"], g["q"], surf, info, g["u"], g["uold"], steps, prec)
        with gpu_ibm_block(cfg, g["coords"], g["nvert"], g["q"], surf, info, g["u"], g["uold"], prec) as b:
            b.RungeKutta(steps)
            want = b.Q()
        want_if = _single_iface(cfg, steps, prec)
        if prec == "fp64":
            assert max(per_field_rel_l2(got, g["q_steps"])) <= RTOL_L2
            assert np.array_equal(got, want), max(per_field_rel_l2(got, want))
            assert np.array_equal(got_if, want_if)
        else:
            assert max(per_field_rel_l2(got, want)) <= 1e-7
            assert max(per_field_rel_l2(got_if, want_if)) <= 1e-7


def test_synthetic_list_on_a_coded_block_equals_single_block():
    """A synthetic list (chained donors, duplicate nodes, entries without an
    element, a moving surface) on a block with slip and no-slip walls and
    inflow/outflow, 3 steps."""
    n = (31, 23, 27)
    coords = W.periodic_grid(n, 2 * np.pi, amp=0.04)
    shape = coords.shape[:3]
    cfg = O.Config(mx=n[0] + 2, my=n[1] + 2, mz=n[2] + 2, bctype=(3, 3, 1, 1, 45, 44), immersed=1, les=1,
                   inviscid=0, fluxorder=3, ren=500., ma=0.3, pr=0.71, dt=0.002, isothermal=1, s_x=0.4, s_y=0.7,
                   s_z=0.9)
    surf = W.sphere_surface(2.0, coords[shape[0] // 2, shape[1] // 2, shape[2] // 2], 2)
    info = synthetic_ibm_list(cfg, coords, len(surf["nv1"]), seed=7, radius=6.0)
    rng = np.random.default_rng(7)
    u = rng.normal(size=(len(surf["x"]), 3)) * 0.02
    uold = u * 0.99
    q = W.random_smooth_state(shape, seed=13, periodic=False)
    nv = np.zeros(shape)
    nv[info["nk"], info["nj"], info["ni"]] = 1.0
    got, _ = _run_batch(cfg, coords, nv, q, surf, info, u, uold, 3)
    with gpu_ibm_block(cfg, coords, nv, q, surf, info, u, uold) as b:
        b.RungeKutta(3)
        want = b.Q()
    assert np.isfinite(got).all()
    assert np.array_equal(got, want), max(per_field_rel_l2(got, want))


def test_immersed_list_errors():
    from chimera_comp_les_b200._lib import CB_E_STATE, CB_E_UNSUPPORTED, ChimeraError
    from chimera_comp_les_b200.batch import Batch
    cfg, meta, g, info, surf = load_ibm_golden("sphere_kflow45")
    dims = [(cfg.mx, cfg.my, cfg.mz), IFACE]
    with Batch(dims, **_batch_kwargs(cfg)) as bt:
        bt.set_ibm_surface(0, surf)
        with pytest.raises(ChimeraError) as e:  # block 0 has no face codes yet
            bt.set_ibm_list(0, 0, info, g["coords"])
        assert e.value.code == CB_E_UNSUPPORTED
        bt.set_bctype(0, tuple(cfg.bctype))
        bt.set_ibm_list(0, 0, info, g["coords"])
        with pytest.raises(ChimeraError) as e:  # a block with a list keeps its codes
            bt.set_bctype(0, (7,) * 6)
        assert e.value.code == CB_E_STATE
        with pytest.raises(ChimeraError) as e:  # and its periodic directions (the list's donors)
            bt.set_bctype(0, (3, 3, 7, 7, 45, 45))
        assert e.value.code == CB_E_STATE
        with pytest.raises(ChimeraError) as e:
            bt.set_ibm_options(0, 1)  # -wallfunction 1 is not built
        assert e.value.code == CB_E_UNSUPPORTED
