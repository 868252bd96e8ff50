"""GPU parity: the CUDA path (through the C-ABI) against the reference's own
outputs (golden fixtures) and against the oracle restatement.

Bar (FP64 form): per conserved field, relative L2 <= 1e-12 (RTOL_L2).
"""
import numpy as np
import pytest

import oracle as O
from chimera_comp_les_b200 import ChimeraError
from chimera_comp_les_b200 import workloads as W

from _common import RTOL_L2, golden_names, gpu_block, load_golden, oracle_run, per_field_rel_l2

pytestmark = pytest.mark.gpu

NAMES = golden_names()


def _setup(cfg, coords, q, nvert):
    b = gpu_block(cfg)
    b.FormMetrics(coords)
    b.set_nvert(nvert)
    b.SetInitialCondition(q)
    return b


@pytest.mark.parametrize("name", NAMES)
def test_device_metrics_match_reference(name):
    cfg, meta, g = load_golden(name)
    with _setup(cfg, g["coords"], g["q"], g["nvert"]) as b:
        csi, eta, zet, aj = b.metrics()
    for k, got in (("csi", csi), ("eta", eta), ("zet", zet), ("aj", aj)):
        ref = g["metrics_" + k].reshape(got.shape)
        assert O.rel_l2(got, ref) <= 1e-14, k


@pytest.mark.parametrize("name", NAMES)
def test_rhs_matches_reference(name):
    cfg, meta, g = load_golden(name)
    with _setup(cfg, g["coords"], g["q"], g["nvert"]) as b:
        if cfg.les and not cfg.inviscid:
            b.CalcUCat()
            b.Compute_eddy_viscosity_LES()
            nut = b.nu_t()
            assert O.rel_l2(nut, g["nut"]) <= RTOL_L2
        rhs = b.formRHS(0)
    errs = per_field_rel_l2(rhs, g["rhs"])
    assert max(errs) <= RTOL_L2, errs


@pytest.mark.parametrize("name", NAMES)
def test_time_steps_match_reference(name):
    cfg, meta, g = load_golden(name)
    with _setup(cfg, g["coords"], g["q"], g["nvert"]) as b:
        b.RungeKutta(meta["steps"])
        q = b.Q()
    errs = per_field_rel_l2(q, g["q_steps"])
    assert max(errs) <= RTOL_L2, errs


# Odd sizes: several tiles in i and j, several k chunks, partial tiles.
ORACLE_CASES = [
    ("les_visc_muscl", (37, 21, 26), dict(les=1, inviscid=0, fluxorder=2, ren=1600., ma=0.1, pr=0.71, dt=0.002), False),
    ("les_visc_weno_mask", (33, 17, 23), dict(les=1, inviscid=0, fluxorder=3, s_x=0.2, s_y=0.5, s_z=0.9, ren=500., ma=0.3, pr=0.71, dt=0.002), True),
    ("std_visc_weno_mask", (35, 41, 20), dict(les=0, inviscid=0, fluxorder=3, ren=500., ma=0.3, pr=0.71, dt=0.002), True),
    ("std_inv_muscl", (40, 12, 31), dict(les=0, inviscid=1, fluxorder=2, dt=0.002), False),
    # nvert values that are not multiples of 1/4: the kernel reads nvert from
    # global memory instead of its shared-memory byte code
    ("les_visc_weno_mask_offgrid", (33, 17, 23), dict(les=1, inviscid=0, fluxorder=3, ren=500., ma=0.3, pr=0.71, dt=0.002), "offgrid"),
    ("std_visc_weno_mask_offgrid", (35, 21, 20), dict(les=0, inviscid=0, fluxorder=3, ren=500., ma=0.3, pr=0.71, dt=0.002), "offgrid"),
    # multiples of 1/4 around every threshold (0.1, 0.5, 2.9, 7): byte-code path
    ("les_visc_weno_mask_quarters", (33, 17, 23), dict(les=1, inviscid=0, fluxorder=3, ren=500., ma=0.3, pr=0.71, dt=0.002), "quarters"),
]


def _mask(shape, seed, kind=True):
    """Three spheres: band 1 / solid 3 (the reference's IBM encoding), or with
    "offgrid" values 0.3 / 0.6 / 2.95 / 7.3 and "quarters" 0.25 / 0.75 / 3.0 / 7.25."""
    rng = np.random.default_rng(seed)
    mz, my, mx = shape
    z, y, x = np.meshgrid(np.arange(mz), np.arange(my), np.arange(mx), indexing="ij")
    vals = {True: (1.0, 1.0, 3.0, 3.0), "offgrid": (0.3, 0.6, 2.95, 7.3), "quarters": (0.25, 0.75, 3.0, 7.25)}[kind]
    nv = np.zeros(shape)
    for _ in range(3):
        c = rng.uniform(4, np.array([mx, my, mz]) - 4)
        r = np.sqrt((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2)
        for rad, v in zip((3.2, 2.6, 1.9, 1.2), vals):
            nv[r < rad] = np.maximum(nv[r < rad], v)
    return nv


@pytest.mark.parametrize("name,n,kw,mask", ORACLE_CASES, ids=[c[0] for c in ORACLE_CASES])
def test_rhs_and_steps_match_oracle(name, n, kw, mask):
    coords = W.periodic_grid(n, 2 * np.pi, amp=0.04)
    shape = coords.shape[:3]
    cfg = O.Config(mx=n[0] + 2, my=n[1] + 2, mz=n[2] + 2, **kw)
    q = W.random_smooth_state(shape, seed=11)
    nv = _mask(shape, 5, mask) if mask else np.zeros(shape)
    ref = oracle_run(cfg, coords, q, nv, steps=2)
    with _setup(cfg, coords, q, nv) as b:
        if cfg.les and not cfg.inviscid:
            b.CalcUCat()
            b.Compute_eddy_viscosity_LES()
            assert O.rel_l2(b.nu_t(), ref["nut"]) <= RTOL_L2
        rhs = b.formRHS(0)
        assert max(per_field_rel_l2(rhs, ref["rhs"])) <= RTOL_L2
    with _setup(cfg, coords, q, nv) as b:
        b.RungeKutta(2)
        assert max(per_field_rel_l2(b.Q(), ref["q_steps"])) <= RTOL_L2


def test_tgv_full_size_parity():
    """Viscous LES of the compressible TGV at 128^3 (m = 130^3), curvilinear
    perturbed grid: one RHS and one time step against the oracle."""
    n = 128
    coords = W.periodic_grid(n, 2 * np.pi, amp=0.05)
    cfg = O.Config(mx=n + 2, my=n + 2, mz=n + 2, les=1, inviscid=0, fluxorder=2, ren=1600., ma=0.1,
                   pr=0.71, gamma=1.4, dt=1e-3)
    q = W.tgv_state(coords, gamma=1.4, ma=0.1)
    nv = np.zeros(coords.shape[:3])
    ref = oracle_run(cfg, coords, q, nv, steps=1)
    with _setup(cfg, coords, q, nv) as b:
        b.CalcUCat()
        b.Compute_eddy_viscosity_LES()
        rhs = b.formRHS(0)
    assert max(per_field_rel_l2(rhs, ref["rhs"])) <= RTOL_L2
    with _setup(cfg, coords, q, nv) as b:
        b.RungeKutta(1)
        q1 = b.Q()
    assert max(per_field_rel_l2(q1, ref["q_steps"])) <= RTOL_L2


def test_graph_replay_equals_eager_launches():
    n = (30, 20, 18)
    coords = W.periodic_grid(n, 2 * np.pi, amp=0.05)
    cfg = O.Config(mx=n[0] + 2, my=n[1] + 2, mz=n[2] + 2, les=1, inviscid=0, fluxorder=3, ren=800., ma=0.2,
                   pr=0.71, dt=0.002)
    q = W.random_smooth_state(coords.shape[:3], seed=3)
    nv = np.zeros(coords.shape[:3])
    with _setup(cfg, coords, q, nv) as b:
        b.RungeKutta(7)  # graphs captured and replayed
        qa = b.Q()
    with _setup(cfg, coords, q, nv) as b:
        b.timing(True)   # timing forces eager launches
        b.RungeKutta(7)
        qb = b.Q()
    assert np.array_equal(qa, qb)


def test_nonfinite_state_reports_status_not_fault():
    """Host-side fault injection: a NaN in the uploaded state makes the step
    report CB_E_NONFINITE through the device status word."""
    n = (16, 12, 10)
    coords = W.periodic_grid(n, 2 * np.pi)
    cfg = O.Config(mx=n[0] + 2, my=n[1] + 2, mz=n[2] + 2, les=0, inviscid=1, fluxorder=2, dt=0.001)
    q = W.random_smooth_state(coords.shape[:3], seed=1)
    q[5, 6, 7, 4] = np.nan
    with _setup(cfg, coords, q, np.zeros(coords.shape[:3])) as b:
        with pytest.raises(ChimeraError) as ei:
            b.RungeKutta(1)
        assert ei.value.code == 4
        # the context stays usable after the error
        b.SetInitialCondition(W.random_smooth_state(coords.shape[:3], seed=2))
        b.RungeKutta(1)


def test_unsupported_options_fail_loudly():
    # a direction periodic on one face only; WENO5 without the WENO path (fluxorder 2)
    for kw in (dict(bctype=(7, 3, 7, 7, 7, 7)), dict(fluxorder=2, weno_order=5), dict(weno_order=4)):
        with pytest.raises(ChimeraError):
            gpu_block(O.Config(mx=12, my=12, mz=12, **kw))


def test_autotune_changes_launch_shape_not_results():
    """cb_autotune picks the k-chunk by timing; the state it leaves and every
    later step are bit-for-bit those of the untuned context."""
    n = (40, 30, 36)
    coords = W.periodic_grid(n, 2 * np.pi, amp=0.04)
    shape = coords.shape[:3]
    cfg = O.Config(mx=n[0] + 2, my=n[1] + 2, mz=n[2] + 2, les=1, inviscid=0, fluxorder=3, ren=1600., ma=0.1,
                   pr=0.71, dt=0.002)
    q = W.random_smooth_state(shape, seed=3)
    nv = np.zeros(shape)
    with _setup(cfg, coords, q, nv) as b:
        b.RungeKutta(2)
        want = b.Q()
    with _setup(cfg, coords, q, nv) as b:
        b.RungeKutta(1)
        before = b.Q()
        best, times = b.autotune()
        assert best in times and all(t > 0 for t in times.values())
        assert np.array_equal(b.Q(), before)
        b.RungeKutta(1)
        assert np.array_equal(b.Q(), want)


SEG_CASES = [
    ("fp64_les_periodic", "fp64", dict(les=1, s_x=0.5, s_y=0.5, s_z=0.5), (40, 30, 36), False),
    ("mixed_les_central", "mixed", dict(les=1), (37, 29, 33), False),
    ("fp64_mask_walls", "fp64", dict(les=1, bctype=(7, 7, 3, 3, 44, 44)), (33, 26, 30), True),
    ("mixed_inviscid_mask", "mixed", dict(les=0, inviscid=1), (35, 17, 41), True),
]


@pytest.mark.parametrize("name,prec,kw,n,mask", SEG_CASES, ids=[c[0] for c in SEG_CASES])
def test_balanced_segments_equal_k_chunks(name, prec, kw, n, mask):
    """k-chunk 0 (balanced segments: ranges of tile-column planes, pieces that
    start mid-column and span columns) gives the results of the chunked grid:
    bit for bit in the FP64 form; in the mixed form (FMA contraction) the
    first k-face of a chunk comes from a second inlined copy of the face code,
    whose FP32 rounding may differ in the last bit, so there the bar is 1e-7."""
    coords = W.periodic_grid(n, 2 * np.pi, amp=0.04)
    shape = coords.shape[:3]
    base = dict(inviscid=0, fluxorder=3, ren=900., ma=0.3, pr=0.71, dt=0.002)
    base.update(kw)
    cfg = O.Config(mx=n[0] + 2, my=n[1] + 2, mz=n[2] + 2, **base)
    q = W.isotropic_turbulence(n, seed=6, k_peak=3.0, mach_t=0.3)
    nv = _mask(shape, 11, True) if mask else np.zeros(shape)
    out = []
    for cand in ([7], [0]):
        with gpu_block(cfg, prec) as b:
            b.FormMetrics(coords)
            b.set_nvert(nv)
            b.SetInitialCondition(q)
            best, _ = b.autotune(cand)
            assert best == cand[0]
            rhs = b.formRHS(0)
            b.RungeKutta(3)
            out.append((rhs, b.Q()))
    if prec == "fp64":
        assert np.array_equal(out[0][0], out[1][0])
        assert np.array_equal(out[0][1], out[1][1])
    else:
        assert max(per_field_rel_l2(out[0][0], out[1][0])) <= 1e-7
        assert max(per_field_rel_l2(out[0][1], out[1][1])) <= 1e-7
