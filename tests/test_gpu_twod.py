"""GPU parity of -twoD 1 (no i-face fluxes, zero x-momentum right-hand side,
lUcat x = 0; rhs.c:1349, 1487, 2135, 2646, 3168, 3465, 4215) against the
oracle restatement, itself bit-exact against the reference
(test_oracle_vs_reference.py::test_twoD1_bitexact_vs_reference).

Bar: FP64 form relative L2 <= 1e-12 (RTOL_L2) per conserved field; mixed form
<= 1e-5; a self-periodic batch bit for bit as the single block."""
import numpy as np
import pytest

import oracle as O
from chimera_comp_les_b200 import workloads as W

from _common import RTOL_L2, gpu_block, oracle_run, per_field_rel_l2
from test_gpu_parity import _mask

pytestmark = pytest.mark.gpu

CASES = [
    ("les_periodic_mask", dict(les=1, fluxorder=3, ren=800.), True),
    ("dns_iso1_walls", dict(les=0, fluxorder=2, ren=500., isothermal=1, bctype=(7, 7, 1, 1, 7, 7)), False),
    ("les_iso2_walls", dict(les=1, fluxorder=3, ren=400., isothermal=2, twall=1.1, s_x=0.6, s_y=0.6, s_z=0.6,
                            bctype=(7, 7, 1, 1, 7, 7)), False),
]


@pytest.mark.parametrize("name,kw,mask", CASES, ids=[c[0] for c in CASES])
def test_twoD1_matches_oracle(name, kw, mask):
    n = (37, 29, 33)
    coords = W.periodic_grid(n, 2 * np.pi, amp=0.04)
    shape = coords.shape[:3]
    cfg = O.Config(mx=n[0] + 2, my=n[1] + 2, mz=n[2] + 2, inviscid=0, ma=0.3, pr=0.71, dt=0.002, twoD=1, **kw)
    q = W.random_smooth_state(shape, seed=11, periodic=False) if cfg.bctype[2] != 7 else \
        W.isotropic_turbulence(n, seed=11, k_peak=3.0, mach_t=0.3)
    nv = _mask(shape, 6, True) if mask else np.zeros(shape)
    want = oracle_run(cfg, coords, q, nv, steps=3)
    for prec, tol in (("fp64", RTOL_L2), ("mixed", 1e-5)):
        with gpu_block(cfg, prec) as b:
            b.FormMetrics(coords)
            b.set_nvert(nv)
            b.SetInitialCondition(q)
            b.RungeKutta(3)
            errs = per_field_rel_l2(b.Q(), want["q_steps"])
        assert max(errs) <= tol, (prec, errs)
    with gpu_block(cfg) as b:
        b.FormMetrics(coords)
        b.set_nvert(nv)
        b.SetInitialCondition(q)
        if cfg.les:
            b.CalcUCat()
            b.Compute_eddy_viscosity_LES()
        rhs = b.formRHS(0)
    assert max(per_field_rel_l2(rhs, want["rhs"])) <= RTOL_L2
    assert not np.any(rhs[1:-1, 1:-1, 1:-1, 1])


def test_twoD1_batch_equals_single_block():
    from chimera_comp_les_b200 import Block
    from chimera_comp_les_b200.batch import Batch
    dims = [(26, 22, 20), (30, 18, 24)]
    opts = dict(les=1, inviscid=0, fluxorder=3, ren=1600., ma=0.1, pr=0.71, dt=2e-3, twod=1)
    inputs = []
    for b, d in enumerate(dims):
        n = (d[0] - 2, d[1] - 2, d[2] - 2)
        inputs.append((W.periodic_grid(n, 2 * np.pi, amp=0.03),
                       W.isotropic_turbulence(n, 30 + b, k_peak=3.0, mach_t=0.3)))
    with Batch(dims, **opts) as bt:
        for k, (coords, q) in enumerate(inputs):
            bt.FormMetrics(k, coords)
            bt.SetInitialCondition(k, q)
        bt.halo_periodic()
        bt.RungeKutta(3)
        got = [bt.Q(k) for k in range(len(dims))]
    for d, (coords, q), g in zip(dims, inputs, got):
        with Block(*d, **opts) as blk:
            blk.FormMetrics(coords)
            blk.SetInitialCondition(q)
            blk.RungeKutta(3)
            assert np.array_equal(g, blk.Q())
