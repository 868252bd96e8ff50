"""CFL time step on the GPU (cb_cfl_dt): warp-shuffle max reduction of the
convective spectral radius, against its host twin in numpy."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,solid", [((30, 26, 22), False), ((41, 33, 29), True)])
def test_cfl_dt_matches_host(n, solid):
    from chimera_comp_les_b200 import Block
    from chimera_comp_les_b200 import diagnostics as D
    from chimera_comp_les_b200 import workloads as W
    coords = W.distorted_periodic_grid(n, 2 * math.pi, 0.03, seed=4)
    q = W.isotropic_turbulence(n, 9, k_peak=3.0, mach_t=0.4)
    nv = np.zeros(q.shape[:3])
    if solid:  # a solid slab and an interface band carry no RHS and are skipped
        nv[:, 5:9, 7:12] = 1.0
        nv[:, 4, 7:12] = 0.5
    with Block(n[0] + 2, n[1] + 2, n[2] + 2, les=1, fluxorder=3) as blk:
        blk.FormMetrics(coords)
        blk.set_nvert(nv)
        blk.SetInitialCondition(q)
        dt, lam = blk.cfl_dt(0.5)
        csi, eta, zet, aj = blk.metrics()
    want = D.spectral_radius_max(q, csi, eta, zet, aj, nv)
    assert lam > 0
    assert abs(lam - want) <= 1e-14 * want, (lam, want)
    assert dt == pytest.approx(0.5 / want, rel=1e-14)
