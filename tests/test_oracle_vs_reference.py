"""Live pin: oracle restatement vs the reference's own code (oracle/_ref),
on seeded inputs beyond the committed fixtures.  Skipped where neither the
prebuilt oracle/_ref library nor the reference sources are present."""
import itertools

import numpy as np
import pytest

import oracle as O
from chimera_comp_les_b200 import workloads as W

pytestmark = pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) not available")


def _nvert(shape, seed):
    rng = np.random.default_rng(seed)
    mz, my, mx = shape
    z, y, x = np.meshgrid(np.arange(mz), np.arange(my), np.arange(mx), indexing="ij")
    c = rng.uniform(4, min(shape) - 4, 3)
    r = np.sqrt((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2)
    nv = np.zeros(shape)
    nv[r < 2.6] = 1.0
    nv[r < 1.7] = 3.0
    return nv


CASES = list(itertools.product([0, 1], [0, 1], [1, 2, 3], [0, 1]))


@pytest.mark.parametrize("les,inv,fo,mask", CASES)
def test_restatement_bitexact_vs_reference(les, inv, fo, mask):
    n = (12, 13, 11)
    coords = W.periodic_grid(n, 2 * np.pi, amp=0.05)
    shape = coords.shape[:3]
    cfg = O.Config(mx=n[0] + 2, my=n[1] + 2, mz=n[2] + 2, les=les, inviscid=inv, fluxorder=fo,
                   s_x=0.4 if les else 1.0, s_y=0.7, s_z=0.9, ren=250., ma=0.3, pr=0.71, dt=0.004)
    q = W.random_smooth_state(shape, seed=7 + fo)
    nv = _nvert(shape, 3) if mask else np.zeros(shape)
    ref = O.RefOracle(cfg, coords)
    ref.set_nvert(nv)
    ref.set_state(q)
    ora = O.Oracle(cfg)
    met = ora.metrics(O.to_padded(cfg, coords))
    nvp = ora.fill_ghosts(O.to_padded(cfg, nv))
    st = ora.initial_state(q)
    nut = ora.zeros(1)
    if les and not inv:
        ref.calc_ucat()
        ref.eddy_viscosity()
        ora.eddy_viscosity(st["q"], met, nvp, nut)
        assert np.array_equal(O.from_padded(nut)[..., 0], ref.nut())
    r_ref = ref.rhs(0)
    r_ora = O.from_padded(ora.rhs(st["q"], met, nvp, nut, ora.sigma() if les else None))
    assert np.array_equal(r_ora, r_ref)
    ref2 = O.RefOracle(cfg, coords)
    ref2.set_nvert(nv)
    ref2.set_state(q)
    ref2.steps(2)
    st = ora.initial_state(q)
    ora.steps(2, st, met, nvp)
    assert np.array_equal(O.from_padded(st["q"]), ref2.Q())
