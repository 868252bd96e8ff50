"""The constant-blend variants of the stage kernel.

With the sensor off, formConvectionLES blends (1 - sigma) * upwind +
sigma * central with sigma = s_x = s_y = s_z on every face (rhs.c:3549-3560).
When that value is exactly 1 or 0 the kernel skips the part multiplied by
zero.  Bar: bit-for-bit the general blend in the FP64 form (a block whose
nvert holds one fluid value 0.05 runs the general kernel and changes no
arithmetic: every nvert threshold of the path is >= 0.1), and the oracle at
RTOL_L2; the mixed form within 1e-6 of its general kernel."""
import numpy as np
import pytest

import oracle as O
from chimera_comp_les_b200 import workloads as W

from _common import RTOL_L2, gpu_block, per_field_rel_l2

pytestmark = pytest.mark.gpu

CASES = [
    ("central_rusanov", 1.0, 0),
    ("central_roe", 1.0, 1),
    ("upwind_rusanov", 0.0, 0),
    ("upwind_roe", 0.0, 1),
]


def _run(cfg, coords, q, nv, precision, steps):
    with gpu_block(cfg, precision) as b:
        b.FormMetrics(coords)
        b.set_nvert(nv)
        b.SetInitialCondition(q)
        b.RungeKutta(steps)
        return b.Q()


@pytest.mark.parametrize("name,sig,flux", CASES, ids=[c[0] for c in CASES])
def test_constant_sigma_variant_equals_general_blend(name, sig, flux):
    n = (37, 29, 33)
    coords = W.periodic_grid(n, 2 * np.pi, amp=0.04)
    shape = coords.shape[:3]
    cfg = O.Config(mx=n[0] + 2, my=n[1] + 2, mz=n[2] + 2, les=1, inviscid=0, fluxorder=3, ren=900., ma=0.3,
                   pr=0.71, dt=0.002, s_x=sig, s_y=sig, s_z=sig, flux=flux)
    q = W.isotropic_turbulence(n, seed=4, k_peak=3.0, mach_t=0.3)
    zero = np.zeros(shape)
    marked = zero.copy()
    marked[shape[0] // 2, shape[1] // 2, shape[2] // 2] = 0.05
    fast = {}
    for prec in ("fp64", "mixed"):
        fast[prec] = _run(cfg, coords, q, zero, prec, 4)
        general = _run(cfg, coords, q, marked, prec, 4)
        if prec == "fp64":
            assert np.array_equal(fast[prec], general)
        else:
            assert max(per_field_rel_l2(fast[prec], general)) <= 1e-6
    if flux == 0:  # Rusanov: the reference's flux
        o = O.Oracle(cfg)
        met = o.metrics(o.fill_ghosts(O.to_padded(cfg, coords)))
        st = o.initial_state(q)
        o.steps(4, st, met, o.fill_ghosts(O.to_padded(cfg, zero)))
        assert max(per_field_rel_l2(fast["fp64"], O.from_padded(st["q"]))) <= RTOL_L2
