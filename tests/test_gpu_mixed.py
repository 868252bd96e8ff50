"""Mixed-precision form (FP32 reconstruction/flux/viscous/SGS arithmetic,
FP64 state, EOS, metrics and RK combination) against the FP64 forms.

Bars: one RHS on an O(1) random state within relative L2 1e-5 per field of
the oracle; the TGV after 100 steps within relative L2 1e-5 per field of the
FP64 GPU form (the stated error of the mixed-vs-FP64 metric)."""
import numpy as np
import pytest

import oracle as O
from chimera_comp_les_b200 import Block
from chimera_comp_les_b200 import workloads as W

from _common import gpu_block, oracle_run, per_field_rel_l2

pytestmark = pytest.mark.gpu

MIXED_RHS_RTOL = 1e-5
MIXED_STEPS_RTOL = 1e-5


@pytest.mark.parametrize("fluxorder,mask", [(2, False), (3, True)])
def test_mixed_rhs_close_to_oracle(fluxorder, mask):
    n = (33, 17, 23)
    coords = W.periodic_grid(n, 2 * np.pi, amp=0.04)
    shape = coords.shape[:3]
    cfg = O.Config(mx=n[0] + 2, my=n[1] + 2, mz=n[2] + 2, les=1, inviscid=0, fluxorder=fluxorder, s_x=0.7,
                   s_y=0.8, s_z=0.9, ren=1600., ma=0.1, pr=0.71, dt=0.002)
    q = W.random_smooth_state(shape, seed=12)
    nv = np.zeros(shape)
    if mask:
        nv[10:14, 7:11, 14:19] = 3.0
    ref = oracle_run(cfg, coords, q, nv)
    with gpu_block(cfg, "mixed") as b:
        b.FormMetrics(coords)
        b.set_nvert(nv)
        b.SetInitialCondition(q)
        b.CalcUCat()
        b.Compute_eddy_viscosity_LES()
        rhs = b.formRHS(0)
    errs = per_field_rel_l2(rhs, ref["rhs"])
    assert max(errs) <= MIXED_RHS_RTOL, errs


@pytest.mark.parametrize("n", [64, 128])
def test_mixed_tgv_100_steps_within_1e5_of_fp64(n):
    coords = W.periodic_grid(n, 2 * np.pi, amp=0.05)
    q0 = W.tgv_state(coords)
    out = {}
    for prec in ("fp64", "mixed"):
        with Block(n + 2, n + 2, n + 2, les=1, fluxorder=3, ren=1600., ma=0.1, pr=0.71, dt=2e-3, precision=prec) as b:
            b.FormMetrics(coords)
            b.set_nvert(np.zeros(coords.shape[:3]))
            b.SetInitialCondition(q0)
            b.RungeKutta(100)
            out[prec] = b.Q()
    errs = per_field_rel_l2(out["mixed"], out["fp64"])
    assert max(errs) <= MIXED_STEPS_RTOL, errs
