"""Non-periodic boundary codes on the GPU (FormBCS rhs.c:477-1227 and the wall
branches of formConvection / formViscous): RHS and RK steps against the oracle
restatement, which is bit-exact against the reference
(tests/test_oracle_vs_reference.py::test_formbcs_restatement_bitexact_vs_reference)."""
import numpy as np
import pytest

import oracle as O
from _common import RTOL_L2, gpu_block, oracle_run, per_field_rel_l2
from chimera_comp_les_b200 import workloads as W

pytestmark = pytest.mark.gpu

BC = [(3, 3, 1, 1, 45, 44), (7, 7, 1, 1, 7, 7), (3, 3, 3, 3, 55, 45), (51, 51, 10, 10, 51, 51),
      (3, 3, 1, 1, 44, 49), (7, 7, 3, 3, 45, 8), (1, 1, 1, 1, 44, 45)]


@pytest.mark.parametrize("bct", BC)
@pytest.mark.parametrize("les,iso,fo", [(0, 0, 3), (1, 1, 3), (0, 1, 2)])
def test_boundary_codes_match_oracle(bct, les, iso, fo):
    n = (35, 17, 23)  # several tiles in i and j, partial tiles
    coords = W.periodic_grid(n, 2 * np.pi, amp=0.04)
    shape = coords.shape[:3]
    cfg = O.Config(mx=n[0] + 2, my=n[1] + 2, mz=n[2] + 2, bctype=bct, les=les, inviscid=0, fluxorder=fo,
                   isothermal=iso, s_x=0.4 if les else 1.0, s_y=0.7, s_z=0.9, ren=250., ma=0.3, pr=0.71, dt=0.002)
    q = W.random_smooth_state(shape, seed=9, periodic=False)
    nv = np.zeros(shape)
    ref = oracle_run(cfg, coords, q, nv, steps=3)
    with gpu_block(cfg) as b:
        b.FormMetrics(coords)
        b.set_nvert(nv)
        b.SetInitialCondition(q)
        if cfg.les:
            b.CalcUCat()
            b.Compute_eddy_viscosity_LES()
            assert O.rel_l2(b.nu_t(), ref["nut"]) <= RTOL_L2
        rhs = b.formRHS(0)
    assert max(per_field_rel_l2(rhs, ref["rhs"])) <= RTOL_L2
    with gpu_block(cfg) as b:
        b.FormMetrics(coords)
        b.set_nvert(nv)
        b.SetInitialCondition(q)
        b.RungeKutta(3)
        got = b.Q()
    assert max(per_field_rel_l2(got, ref["q_steps"])) <= RTOL_L2
    with gpu_block(cfg, precision="mixed") as b:
        b.FormMetrics(coords)
        b.set_nvert(nv)
        b.SetInitialCondition(q)
        b.RungeKutta(3)
        assert max(per_field_rel_l2(b.Q(), ref["q_steps"])) <= 1e-5


ISO2_BC = [(3, 3, 1, 1, 45, 44), (7, 7, 1, 1, 7, 7), (1, 1, 1, 1, 44, 45)]


@pytest.mark.parametrize("bct", ISO2_BC)
@pytest.mark.parametrize("les,twoD,twall", [(0, 0, 1.0), (1, 1, 1.2)])
def test_characteristic_isothermal_walls_match_oracle(bct, les, twoD, twall):
    """-isothermal 2 on the j walls (code 1): the characteristic wall of
    Poinsot & Lele (rhs.c:663-733 low, 803-818 high), with -twoD and -Twall."""
    n = (35, 17, 23)
    coords = W.periodic_grid(n, 2 * np.pi, amp=0.04)
    shape = coords.shape[:3]
    cfg = O.Config(mx=n[0] + 2, my=n[1] + 2, mz=n[2] + 2, bctype=bct, les=les, inviscid=0, fluxorder=3,
                   isothermal=2, twoD=twoD, twall=twall, s_x=0.4 if les else 1.0, s_y=0.7, s_z=0.9, ren=250.,
                   ma=0.3, pr=0.71, dt=0.002)
    q = W.random_smooth_state(shape, seed=9, periodic=False)
    nv = np.zeros(shape)
    ref = oracle_run(cfg, coords, q, nv, steps=3)
    assert np.isfinite(ref["q_steps"]).all()
    for prec, tol in (("fp64", RTOL_L2), ("mixed", 1e-5)):
        with gpu_block(cfg, precision=prec) as b:
            b.FormMetrics(coords)
            b.set_nvert(nv)
            b.SetInitialCondition(q)
            b.RungeKutta(3)
            assert max(per_field_rel_l2(b.Q(), ref["q_steps"])) <= tol, prec


# with this seeded state, k-hi code 49 behind the 52 inlet on walled j faces
# drives the restatement itself to rho, p < 0 at the outlet, so that pairing
# uses the outflow code 45
INFLOW = [(7, 7, 3, 3, 52, 44), (7, 7, 3, 3, 47, 45), (3, 3, 1, 1, 52, 45), (7, 7, 7, 7, 47, 8)]


@pytest.mark.parametrize("bct", INFLOW)
@pytest.mark.parametrize("les,ti0", [(0, 1), (1, 6)])
def test_inflow_codes_52_47_match_oracle(bct, les, ti0):
    """The k-lo inflow codes that read the node coordinates: the
    characteristic cos^2 inlet 52 (rhs.c:854-874) and the power-law inlet 47
    with perturbations travelling in x and time (rhs.c:904-950), whose step
    index comes from cb_set_time_index (a restart at step ti0 - 1)."""
    n = (35, 17, 23)
    coords = W.periodic_grid(n, 2 * np.pi, amp=0.04)
    coords[..., 1] = 1.5 * coords[..., 1] + 1.0  # y on both sides of 47's y = 8
    shape = coords.shape[:3]
    cfg = O.Config(mx=n[0] + 2, my=n[1] + 2, mz=n[2] + 2, bctype=bct, les=les, inviscid=0, fluxorder=3,
                   s_x=0.4 if les else 1.0, s_y=0.7, s_z=0.9, ren=250., ma=0.3, pr=0.71, dt=0.002, ti0=ti0)
    q = W.random_smooth_state(shape, seed=19, periodic=False)
    nv = np.zeros(shape)
    ref = oracle_run(cfg, coords, q, nv, steps=3)
    qs = ref["q_steps"]
    assert np.isfinite(qs).all()
    ke = 0.5 * (qs[..., 1] ** 2 + qs[..., 2] ** 2 + qs[..., 3] ** 2) / qs[..., 0]
    assert qs[..., 0].min() > 0 and (qs[..., 4] - ke).min() > 0  # a physical case: the device flags rho, p <= 0
    for prec, tol in (("fp64", RTOL_L2), ("mixed", 1e-5)):
        with gpu_block(cfg, precision=prec) as b:
            b.FormMetrics(coords)
            b.set_nvert(nv)
            b.SetInitialCondition(q)
            b.set_time_index(ti0 - 1)
            b.RungeKutta(3)
            assert max(per_field_rel_l2(b.Q(), ref["q_steps"])) <= tol, prec
