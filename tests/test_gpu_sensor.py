"""LES pressure shock sensor (-calc_sigma 1, rhs.c:3328-3433) on the GPU: the
hybrid weights, the RHS and two RK steps against the oracle restatement (itself
bit-exact against the reference, tests/test_oracle_vs_reference.py), and the
mixed form within its bar."""
import numpy as np
import pytest

import oracle as O
from _common import RTOL_L2, gpu_block, oracle_run, per_field_rel_l2
from chimera_comp_les_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _jump_state(shape, seed):
    q = W.random_smooth_state(shape, seed=seed)
    mz, my, mx = shape
    z, y, x = np.meshgrid(np.arange(mz), np.arange(my), np.arange(mx), indexing="ij")
    jump = (x + 0.7 * y + 0.4 * z) > 0.55 * (mx + my + mz) * 0.6
    q[..., 0] = np.where(jump, 1.6 * q[..., 0], q[..., 0])
    q[..., 4] = np.where(jump, 1.9 * q[..., 4], q[..., 4])
    return q


CASES = [
    ("visc", (37, 21, 26), dict(les=1, inviscid=0, fluxorder=3, s_x=0.9, s_y=0.8, s_z=1.0, ren=250., ma=0.3,
                                pr=0.71, dt=0.002, calc_sigma=1)),
    ("inv_min", (33, 40, 19), dict(les=1, inviscid=1, fluxorder=2, s_x=1.0, s_y=1.0, s_z=0.7, dt=0.002, calc_sigma=1,
                                   s_x_min=0.2, s_y_min=0.1, s_z_min=0.3)),
    # -ABC: raw weights 0 above plane k = 15 (rhs.c:3341-3368)
    ("visc_abc", (37, 21, 26), dict(les=1, inviscid=0, fluxorder=3, s_x=0.9, s_y=0.8, s_z=1.0, ren=250., ma=0.3,
                                    pr=0.71, dt=0.002, calc_sigma=1, s_x_min=0.1, s_y_min=0.2, s_z_min=0.05, abc=15)),
]


@pytest.mark.parametrize("name,n,kw", CASES, ids=[c[0] for c in CASES])
def test_sensor_rhs_and_steps_match_oracle(name, n, kw):
    coords = W.periodic_grid(n, 2 * np.pi, amp=0.04)
    shape = coords.shape[:3]
    cfg = O.Config(mx=n[0] + 2, my=n[1] + 2, mz=n[2] + 2, **kw)
    q = _jump_state(shape, 5)
    nv = np.zeros(shape)
    ref = oracle_run(cfg, coords, q, nv, steps=2)
    with gpu_block(cfg) as b:
        b.FormMetrics(coords)
        b.set_nvert(nv)
        b.SetInitialCondition(q)
        if not cfg.inviscid:
            b.CalcUCat()
            b.Compute_eddy_viscosity_LES()
        rhs = b.formRHS(0)
    assert max(per_field_rel_l2(rhs, ref["rhs"])) <= RTOL_L2
    with gpu_block(cfg) as b:
        b.FormMetrics(coords)
        b.set_nvert(nv)
        b.SetInitialCondition(q)
        b.RungeKutta(2)
        assert max(per_field_rel_l2(b.Q(), ref["q_steps"])) <= RTOL_L2
    with gpu_block(cfg, precision="mixed") as b:
        b.FormMetrics(coords)
        b.set_nvert(nv)
        b.SetInitialCondition(q)
        b.RungeKutta(2)
        assert max(per_field_rel_l2(b.Q(), ref["q_steps"])) <= 1e-5

