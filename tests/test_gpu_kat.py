"""Known-answer tests from the mathematics (not from the reference):

* discrete conservation: on a periodic uniform Cartesian box the flux
  differences telescope, so the sum of Rhs/aj over the interior vanishes for
  every conserved field (non-LES scheme: its faces at the periodic seam use
  only the two adjacent nodes, rhs.c:2665-2666);
* the isentropic (Shu) vortex advected on the periodic box [0, 10]^3 with the
  reference's scheme set (inviscid, WENO3 + Rusanov, SSP-RK3): the solution after t is the initial
  vortex translated by t*(1, 1, 0); the error must shrink under refinement.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kw", [dict(les=0, inviscid=1, fluxorder=3), dict(les=0, inviscid=0, fluxorder=2, ren=300.0),
                                dict(les=0, inviscid=0, fluxorder=3, ren=300.0)])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_periodic_box_conserves(kw, precision):
    from chimera_comp_les_b200 import Block
    from chimera_comp_les_b200 import workloads as W
    n = (28, 22, 18)
    coords = W.periodic_grid(n, (2.0, 1.5, 1.25), amp=0.0)
    q = W.random_smooth_state(coords.shape[:3], seed=4, amp=0.1)
    with Block(n[0] + 2, n[1] + 2, n[2] + 2, ma=0.5, pr=0.72, dt=1e-3, precision=precision, **kw) as b:
        b.FormMetrics(coords)
        b.SetInitialCondition(q)
        rhs = b.formRHS(0)
        aj = b.metrics()[3]
    inner = (slice(1, -1),) * 3
    for f in range(5):
        r = rhs[inner + (f,)] / aj[inner]
        scale = np.abs(r).sum()
        if f == 0 and scale == 0:
            continue
        tol = 1e-12 if precision == "fp64" else 1e-5
        assert abs(r.sum()) <= tol * scale, (f, r.sum(), scale)


def _vortex_error(n, t_end):
    from chimera_comp_les_b200 import Block
    from chimera_comp_les_b200 import workloads as W
    L = 10.0
    coords = W.periodic_grid(n, L, amp=0.0)
    q0 = W.vortex_state(coords)
    dx = L / n
    r = q0[..., 0]
    u = np.abs(q0[..., 1] / r) + np.abs(q0[..., 2] / r)
    c = np.sqrt(1.4 * 0.4 * (q0[..., 4] - 0.5 * (q0[..., 1] ** 2 + q0[..., 2] ** 2 + q0[..., 3] ** 2) / r) / r)
    dt0 = 0.5 * dx / float((u + c).max())
    steps = int(math.ceil(t_end / dt0))
    dt = t_end / steps
    with Block(n + 2, n + 2, n + 2, les=0, inviscid=1, fluxorder=3, dt=dt) as b:
        b.FormMetrics(coords)
        b.SetInitialCondition(q0)
        b.RungeKutta(steps)
        q = b.Q()
    shifted = coords.copy()
    shifted[..., 0] = np.mod(coords[..., 0] - t_end, L)
    shifted[..., 1] = np.mod(coords[..., 1] - t_end, L)
    qe = W.vortex_state(shifted)
    inner = (slice(1, -1),) * 3
    d = q[inner + (0,)] - qe[inner + (0,)]
    return float(np.linalg.norm(d) / np.linalg.norm(qe[inner + (0,)] - 1.0)), steps


def test_isentropic_vortex_converges_to_translated_solution():
    e32, _ = _vortex_error(32, 2.0)
    e64, steps = _vortex_error(64, 2.0)
    assert steps > 20
    assert e64 < 0.5 * e32, (e32, e64)
    assert e64 < 0.15, e64
