"""GPU parity of the dynamic Smagorinsky model (-les 2 and its variants,
Compute_Smagorinsky_Constant_1, les.c:134-1472) against the oracle
restatement (itself bit-exact against the reference): the coefficient and the
eddy viscosity after steps, where the recorded CalcUCat state differs from the
current one, on odd sizes with an IBM mask (several tiles and k-chunks).
The reference fixture les2_dynamic_weno_mask runs through test_gpu_parity.

Bar (FP64 form): relative L2 <= 1e-12 (RTOL_L2)."""
import numpy as np
import pytest

import oracle as O
from chimera_comp_les_b200 import ChimeraError
from chimera_comp_les_b200 import workloads as W

from _common import RTOL_L2, gpu_block, per_field_rel_l2
from test_gpu_parity import _mask

pytestmark = pytest.mark.gpu

CASES = [
    ("weno_mask", (37, 29, 33), dict(fluxorder=3, ren=800., max_cs=0.1), True),
    ("muscl_open", (40, 24, 31), dict(fluxorder=2, ren=500., max_cs=0.05), False),
    ("walls_outflow", (33, 26, 30), dict(fluxorder=3, ren=600., max_cs=0.2, bctype=(7, 7, 3, 3, 44, 44)), True),
]


def _case(n, kw, mask):
    coords = W.periodic_grid(n, 2 * np.pi, amp=0.04)
    shape = coords.shape[:3]
    cfg = O.Config(mx=n[0] + 2, my=n[1] + 2, mz=n[2] + 2, les=2, inviscid=0, ma=0.3, pr=0.71, dt=0.002, **kw)
    q = W.random_smooth_state(shape, seed=13)
    nv = _mask(shape, 7, True) if mask else np.zeros(shape)
    return cfg, coords, q, nv


@pytest.mark.parametrize("name,n,kw,mask", CASES, ids=[c[0] for c in CASES])
def test_dynamic_steps_match_oracle(name, n, kw, mask):
    cfg, coords, q, nv = _case(n, kw, mask)
    o = O.Oracle(cfg)
    met = o.metrics(o.fill_ghosts(O.to_padded(cfg, coords)))
    nvp = o.fill_ghosts(O.to_padded(cfg, nv))
    st = o.initial_state(q)
    o.steps(3, st, met, nvp)
    # the coefficient and nu_t of a fourth step's start, from the recorded state
    cs = o.dynamic_smagorinsky(st["q"], st["quc"], met, nvp)
    nut = o.eddy_viscosity_dyn(st["q"], st["quc"], met, nvp, cs, o.zeros(1))
    with gpu_block(cfg) as b:
        b.FormMetrics(coords)
        b.set_nvert(nv)
        b.SetInitialCondition(q)
        b.RungeKutta(3)
        assert max(per_field_rel_l2(b.Q(), O.from_padded(st["q"]))) <= RTOL_L2
        b.Compute_eddy_viscosity_LES()
        cs_d, nut_d = b.CS(), b.nu_t()
    cs_o, nut_o = O.from_padded(cs)[..., 0], O.from_padded(nut)[..., 0]
    assert cs_o.max() > 0.0
    assert O.rel_l2(cs_d, cs_o) <= RTOL_L2
    assert O.rel_l2(nut_d, nut_o) <= RTOL_L2


def test_dynamic_mixed_form_tracks_fp64():
    cfg, coords, q, nv = _case((48, 40, 44), dict(fluxorder=3, ren=1000., max_cs=0.1), False)
    out = {}
    for prec in ("fp64", "mixed"):
        with gpu_block(cfg, prec) as b:
            b.FormMetrics(coords)
            b.set_nvert(nv)
            b.SetInitialCondition(q)
            b.RungeKutta(20)
            out[prec] = b.Q()
    assert max(per_field_rel_l2(out["mixed"], out["fp64"])) <= 1e-5


def test_dynamic_graph_replay_equals_eager():
    cfg, coords, q, nv = _case((30, 22, 26), dict(fluxorder=3, ren=800.), True)
    res = []
    for timing in (False, True):
        with gpu_block(cfg) as b:
            b.FormMetrics(coords)
            b.set_nvert(nv)
            b.SetInitialCondition(q)
            b.timing(timing)
            b.RungeKutta(5)
            res.append(b.Q())
    assert np.array_equal(res[0], res[1])


def test_dynamic_options_are_checked():
    cfg, coords, q, nv = _case((16, 14, 12), dict(fluxorder=3, ren=800.), False)
    with pytest.raises(ChimeraError):
        gpu_block(O.Config(**{**cfg.__dict__, "max_cs": -1.0}))
    with pytest.raises(ChimeraError):
        gpu_block(O.Config(**{**cfg.__dict__, "les": -1}))
    with gpu_block(O.Config(**{**cfg.__dict__, "les": 1})) as b:
        with pytest.raises(ChimeraError):
            b.CS()


VARIANTS = [
    ("les3_pointwise", dict(les=3), False),
    ("testfilter_ik", dict(testfilter_ik=1), True),
    ("i_homo_lines", dict(i_homo_filter=1), True),
    ("ik_homo_planes", dict(i_homo_filter=1, k_homo_filter=1), True),
    ("ijk_homo_box", dict(i_homo_filter=1, j_homo_filter=1, k_homo_filter=1), True),
    ("k_homo_pointwise", dict(k_homo_filter=1), False),
    ("les7_as_local", dict(les=7), False),
    # -twoD 1: the model's in-place lUcat keeps x = rhoU/rho where its loop
    # reached, CalcUCat's x = 0 elsewhere (les.c:234-238, rhs.c:1349)
    ("twoD1", dict(twoD=1), True),
    ("twoD1_ik_homo_planes", dict(twoD=1, i_homo_filter=1, k_homo_filter=1), False),
]


@pytest.mark.parametrize("name,kw,mask", VARIANTS, ids=[v[0] for v in VARIANTS])
def test_dynamic_variants_match_oracle(name, kw, mask):
    """-les 3, -testfilter_ik and the homogeneous filters (i lines, j planes,
    the box) on a turbulent field with several tiles, k-chunks and plane
    reductions: Q after three steps, then Cs and nu_t of the fourth."""
    n = (37, 29, 33)
    coords = W.periodic_grid(n, 2 * np.pi, amp=0.04)
    shape = coords.shape[:3]
    base = dict(les=2, inviscid=0, ma=0.3, pr=0.71, dt=0.002, fluxorder=3, ren=900., max_cs=0.3)
    base.update(kw)
    cfg = O.Config(mx=n[0] + 2, my=n[1] + 2, mz=n[2] + 2, **base)
    q = W.isotropic_turbulence(n, seed=2, k_peak=3.0, mach_t=0.3)
    nv = _mask(shape, 7, True) if mask else np.zeros(shape)
    o = O.Oracle(cfg)
    met = o.metrics(o.fill_ghosts(O.to_padded(cfg, coords)))
    nvp = o.fill_ghosts(O.to_padded(cfg, nv))
    st = o.initial_state(q)
    o.steps(3, st, met, nvp)
    cs = o.dynamic_smagorinsky(st["q"], st["quc"], met, nvp)
    nut = o.eddy_viscosity_dyn(st["q"], st["quc"], met, nvp, cs, o.zeros(1))
    with gpu_block(cfg) as b:
        b.FormMetrics(coords)
        b.set_nvert(nv)
        b.SetInitialCondition(q)
        b.RungeKutta(3)
        assert max(per_field_rel_l2(b.Q(), O.from_padded(st["q"]))) <= RTOL_L2
        b.Compute_eddy_viscosity_LES()
        cs_d, nut_d = b.CS(), b.nu_t()
    cs_o, nut_o = O.from_padded(cs)[..., 0], O.from_padded(nut)[..., 0]
    assert cs_o[nv < 0.1].max() > 0.0  # not every coefficient clipped away
    assert O.rel_l2(cs_d, cs_o) <= RTOL_L2
    assert O.rel_l2(nut_d, nut_o) <= RTOL_L2


def test_les10_matches_oracle():
    """-les 10: the LES right-hand side with nu_t left at zero."""
    n = (30, 22, 26)
    coords = W.periodic_grid(n, 2 * np.pi, amp=0.04)
    cfg = O.Config(mx=n[0] + 2, my=n[1] + 2, mz=n[2] + 2, les=10, inviscid=0, ma=0.3, pr=0.71, dt=0.002,
                   fluxorder=3, ren=900.)
    q = W.isotropic_turbulence(n, seed=3, k_peak=3.0, mach_t=0.3)
    nv = np.zeros(coords.shape[:3])
    o = O.Oracle(cfg)
    met = o.metrics(o.fill_ghosts(O.to_padded(cfg, coords)))
    st = o.initial_state(q)
    o.steps(3, st, met, o.fill_ghosts(O.to_padded(cfg, nv)))
    with gpu_block(cfg) as b:
        b.FormMetrics(coords)
        b.SetInitialCondition(q)
        b.RungeKutta(3)
        assert max(per_field_rel_l2(b.Q(), O.from_padded(st["q"]))) <= RTOL_L2
        assert not np.any(b.nu_t())
