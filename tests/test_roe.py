"""Roe flux with Harten's entropy fix (an upwind flux the reference does not
have): known answers of the CPU restatement, and the GPU against it."""
import math

import numpy as np
import pytest

import oracle as O
from _common import RTOL_L2, gpu_block, oracle_run, per_field_rel_l2
from chimera_comp_les_b200 import workloads as W


def _rhs(cfg, coords, q):
    ora = O.Oracle(cfg)
    met = ora.metrics(O.to_padded(cfg, coords))
    nvp = ora.fill_ghosts(O.to_padded(cfg, np.zeros(q.shape[:3])))
    st = ora.initial_state(q)
    nut = ora.zeros(1)
    return O.from_padded(ora.rhs(st["q"], met, nvp, nut, ora.sigma(st["q"]) if cfg.les else None))


@pytest.mark.parametrize("les", [0, 1])
def test_roe_equals_rusanov_on_a_uniform_state(les):
    """With equal left and right states both fluxes reduce to the physical flux."""
    n = (14, 12, 10)
    coords = W.periodic_grid(n, 2 * np.pi, amp=0.05)
    q = W.conserved(*(np.full(coords.shape[:3], v) for v in (1.2, 0.3, -0.2, 0.1, 0.9)), 1.4)
    kw = dict(mx=n[0] + 2, my=n[1] + 2, mz=n[2] + 2, les=les, inviscid=1, fluxorder=1, dt=0.002)
    a = _rhs(O.Config(flux=0, **kw), coords, q)
    b = _rhs(O.Config(flux=1, **kw), coords, q)
    assert np.array_equal(a, b)


def test_roe_dissipation_differs_from_rusanov_and_reference_refuses_it():
    n = (14, 12, 10)
    coords = W.periodic_grid(n, 2 * np.pi, amp=0.05)
    q = W.random_smooth_state(coords.shape[:3], seed=3)
    kw = dict(mx=n[0] + 2, my=n[1] + 2, mz=n[2] + 2, les=0, inviscid=1, fluxorder=3, dt=0.002)
    a = _rhs(O.Config(flux=0, **kw), coords, q)
    b = _rhs(O.Config(flux=1, **kw), coords, q)
    d = max(per_field_rel_l2(b, a))
    assert np.isfinite(b).all() and d > 1e-6
    with pytest.raises(ValueError):
        O.RefOracle(O.Config(flux=1, **kw), coords)


CASES = [
    ("les_visc", (37, 21, 26), dict(les=1, inviscid=0, fluxorder=3, ren=500., ma=0.3, pr=0.71, dt=0.002)),
    ("std_visc_walls", (35, 17, 23), dict(les=0, inviscid=0, fluxorder=3, bctype=(3, 3, 1, 1, 45, 44), ren=250.,
                                         ma=0.3, pr=0.71, dt=0.002)),
    ("std_inv_muscl", (40, 12, 31), dict(les=0, inviscid=1, fluxorder=2, dt=0.002)),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,n,kw", CASES, ids=[c[0] for c in CASES])
def test_roe_gpu_matches_restatement(name, n, kw):
    coords = W.periodic_grid(n, 2 * np.pi, amp=0.04)
    shape = coords.shape[:3]
    cfg = O.Config(mx=n[0] + 2, my=n[1] + 2, mz=n[2] + 2, flux=1, **kw)
    periodic = all(b == 7 for b in cfg.bctype)
    q = W.random_smooth_state(shape, seed=11, periodic=periodic)
    nv = np.zeros(shape)
    ref = oracle_run(cfg, coords, q, nv, steps=2)
    with gpu_block(cfg) as b:
        b.FormMetrics(coords)
        b.set_nvert(nv)
        b.SetInitialCondition(q)
        if cfg.les:
            b.CalcUCat()
            b.Compute_eddy_viscosity_LES()
        assert max(per_field_rel_l2(b.formRHS(0), ref["rhs"])) <= RTOL_L2
    for prec, tol in (("fp64", RTOL_L2), ("mixed", 1e-5)):
        with gpu_block(cfg, precision=prec) as b:
            b.FormMetrics(coords)
            b.set_nvert(nv)
            b.SetInitialCondition(q)
            b.RungeKutta(2)
            assert max(per_field_rel_l2(b.Q(), ref["q_steps"])) <= tol, prec


@pytest.mark.gpu
def test_roe_vortex_less_dissipative_than_rusanov():
    """Isentropic vortex (inviscid, WENO3, SSP-RK3): Roe's upwinding adds less
    dissipation than Rusanov's, so the translated vortex is closer to exact."""
    from chimera_comp_les_b200 import Block
    n, L, t_end = 48, 10.0, 2.0
    coords = W.periodic_grid(n, L, amp=0.0)
    q0 = W.vortex_state(coords)
    dt = 0.3 * (L / n) / 3.0
    steps = int(math.ceil(t_end / dt))
    dt = t_end / steps
    shifted = coords.copy()
    shifted[..., 0] = np.mod(coords[..., 0] - t_end, L)
    shifted[..., 1] = np.mod(coords[..., 1] - t_end, L)
    qe = W.vortex_state(shifted)
    err = {}
    for flux in ("rusanov", "roe"):
        with Block(n + 2, n + 2, n + 2, les=0, inviscid=1, fluxorder=3, dt=dt, flux=flux) as b:
            b.FormMetrics(coords)
            b.SetInitialCondition(q0)
            b.RungeKutta(steps)
            q = b.Q()
        inner = (slice(1, -1),) * 3
        err[flux] = float(np.linalg.norm(q[inner + (0,)] - qe[inner + (0,)]) / np.linalg.norm(qe[inner + (0,)] - 1))
    assert err["roe"] < err["rusanov"], err
