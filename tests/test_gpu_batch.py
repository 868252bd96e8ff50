"""Batched multi-block form on the GPU (cb_batch_* through the C-ABI).

FP64: every block of a self-periodic batch must evolve bit-for-bit as the
same block alone in a single-block context (itself held to the oracle), in
the persistent form and with one launch per block; sub-blocks of a periodic
box joined by the decomposed halo map must reproduce the undivided box
bit-for-bit.  Mixed form: within the mixed-vs-FP64 bar (relative L2 <= 1e-5).
"""
import math

import numpy as np
import pytest

import oracle as O
from _common import RTOL_L2, oracle_run, per_field_rel_l2

pytestmark = pytest.mark.gpu

OPTS = dict(les=1, inviscid=0, fluxorder=3, eno_order=2, central=2, ren=1600.0, ma=0.1, pr=0.71, gamma=1.4, dt=2e-3)
DIMS = [(26, 22, 20), (34, 18, 24), (20, 30, 16)]


def _inputs(dims, seed0=0):
    from chimera_comp_les_b200 import workloads as W
    out = []
    for b, d in enumerate(dims):
        n = (d[0] - 2, d[1] - 2, d[2] - 2)
        coords = W.distorted_periodic_grid(n, 2 * math.pi, 0.03, seed=seed0 + 10 * b)
        q = W.isotropic_turbulence(n, seed0 + 10 * b + 1, k_peak=3.0, mach_t=0.3)
        out.append((coords, q))
    return out


def _single(d, coords, q, steps, precision="fp64", opts=OPTS):
    from chimera_comp_les_b200 import Block
    with Block(*d, precision=precision, **opts) as blk:
        blk.FormMetrics(coords)
        blk.SetInitialCondition(q)
        blk.RungeKutta(steps)
        return blk.Q()


def _batch(dims, inputs, precision="fp64", opts=OPTS):
    from chimera_comp_les_b200.batch import Batch
    bt = Batch(dims, precision=precision, **opts)
    for k, (coords, q) in enumerate(inputs):
        bt.FormMetrics(k, coords)
        bt.SetInitialCondition(k, q)
    return bt


@pytest.mark.parametrize("per_block", [False, True])
def test_self_periodic_batch_equals_single_blocks(per_block):
    inputs = _inputs(DIMS)
    steps = 3
    with _batch(DIMS, inputs) as bt:
        bt.halo_periodic()
        bt.RungeKutta(steps, per_block=per_block)
        got = [bt.Q(k) for k in range(len(DIMS))]
    for d, (coords, q), g in zip(DIMS, inputs, got):
        want = _single(d, coords, q, steps)
        assert np.array_equal(g, want), max(per_field_rel_l2(g, want))


# the stage-kernel variants of the options: Roe's flux, WENO5-JS (its 32 x 5
# tile and six-plane ring), and the constant blend weights 0 and 1
VARIANTS = [
    ("roe", dict(flux="roe")),
    ("weno5", dict(weno_order=5, s_x=0.5, s_y=0.5, s_z=0.5)),
    ("weno5_roe_sigma0", dict(weno_order=5, flux="roe", s_x=0.0, s_y=0.0, s_z=0.0)),
    ("sigma1", dict(s_x=1.0, s_y=1.0, s_z=1.0)),
    # the shock sensor: per-block weights from the step's input state, each
    # pass followed by the wrap map (with -ABC above plane 9 in the blocks
    # that reach it)
    ("sensor", dict(calc_sigma=1, s_x=0.5, s_y=0.6, s_z=0.7, s_x_min=0.05, sigma_thrsh=1e-4, abc=9)),
    ("sensor_weno5_roe", dict(calc_sigma=1, weno_order=5, flux="roe", s_x=0.8, s_y=0.8, s_z=0.8)),
    # the dynamic Smagorinsky model per block (Germano 27-node means, -les 3
    # pointwise, the homogeneous plane and box means, the -testfilter_ik width)
    ("dynamic", dict(les=2, max_cs=0.1)),
    ("dynamic_les3", dict(les=3, max_cs=0.1)),
    ("dynamic_homo_ik", dict(les=2, i_homo_filter=1, k_homo_filter=1, max_cs=0.1)),
    ("dynamic_box_tf", dict(les=2, i_homo_filter=1, j_homo_filter=1, k_homo_filter=1, testfilter_ik=1, max_cs=0.1)),
    # -les 10: Cs = 0, the eddy viscosity stays zero
    ("les10", dict(les=10)),
]


@pytest.mark.parametrize("per_block", [False, True])
@pytest.mark.parametrize("name,over", VARIANTS, ids=[v[0] for v in VARIANTS])
def test_batch_variants_equal_single_blocks(name, over, per_block):
    """Every option the single-block context builds for the stage kernel runs
    in the batch too: FP64 bit for bit against the same blocks alone, the
    mixed form within 1e-7 of its own single-block runs (with FMA
    contraction a chunk's first k-face may round differently in the last bit
    when the launch shapes differ)."""
    opts = dict(OPTS, **over)
    inputs = _inputs(DIMS, seed0=3)
    steps = 2
    for prec in ("fp64", "mixed"):
        with _batch(DIMS, inputs, precision=prec, opts=opts) as bt:
            bt.halo_periodic()
            bt.RungeKutta(steps, per_block=per_block)
            got = [bt.Q(k) for k in range(len(DIMS))]
        for d, (coords, q), g in zip(DIMS, inputs, got):
            want = _single(d, coords, q, steps, precision=prec, opts=opts)
            if prec == "fp64":
                assert np.array_equal(g, want), max(per_field_rel_l2(g, want))
            else:
                assert max(per_field_rel_l2(g, want)) <= 1e-7


def test_batch_block_matches_oracle():
    """First block of a batch against the CPU restatement (2 steps)."""
    d = (14, 12, 11)
    inputs = _inputs([d, (12, 13, 10)], seed0=5)
    cfg = O.Config(mx=d[0], my=d[1], mz=d[2], **OPTS)
    want = oracle_run(cfg, inputs[0][0], inputs[0][1], np.zeros(inputs[0][1].shape[:3]), steps=2)["q_steps"]
    with _batch([d, (12, 13, 10)], inputs) as bt:
        bt.halo_periodic()
        bt.RungeKutta(2)
        got = bt.Q(0)
    assert max(per_field_rel_l2(got, want)) <= RTOL_L2


def test_python_self_periodic_map_equals_library_map():
    from chimera_comp_les_b200 import batch as B
    inputs = _inputs(DIMS)
    with _batch(DIMS, inputs) as bt:
        bt.set_halo_maps(B.halo_maps_self_periodic(DIMS))
        bt.RungeKutta(2)
        a = [bt.Q(k) for k in range(len(DIMS))]
    with _batch(DIMS, inputs) as bt:
        bt.halo_periodic()
        bt.RungeKutta(2)
        b = [bt.Q(k) for k in range(len(DIMS))]
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def _k_uniform_grid(n, length):
    """Periodic box distorted in x and y only, with a z spacing that is a power
    of two (z differences exact), so the metrics are bit-for-bit independent of
    k and sub-blocks cut along k carry exactly the undivided box's metrics."""
    from chimera_comp_les_b200 import workloads as W
    g = W.periodic_grid(n, length, 0.0)
    sx = 2 * math.pi * g[..., 0] / length[0]
    sy = 2 * math.pi * g[..., 1] / length[1]
    g[..., 0] += 0.04 * np.sin(sy)
    g[..., 1] += 0.03 * np.sin(sx)
    return np.ascontiguousarray(g)


@pytest.mark.parametrize("per_block", [False, True])
def test_decomposed_box_equals_undivided(per_block):
    """k-slabs of a periodic box joined by the decomposed map against the box.

    The reference's 4-point central flux is used only on faces away from the
    block's own boundary layer (pos > 0 && pos < m-2, rhs.c:3483-3547); a cut
    is a block boundary for each slab, so the two agree bit-for-bit only with
    the 2-point central flux (-central 1), used here."""
    from chimera_comp_les_b200 import batch as B
    from chimera_comp_les_b200 import workloads as W
    n = (22, 18, 30)
    M = (n[0] + 2, n[1] + 2, n[2] + 2)
    coords = _k_uniform_grid(n, (2 * math.pi, 2 * math.pi, n[2] * 0.25))
    q = W.isotropic_turbulence(n, 17, k_peak=3.0, mach_t=0.3)
    steps = 3
    opts = dict(OPTS, central=1)
    want = _single(M, coords, q, steps, opts=opts)
    parts = B.decompose(M, [[n[0]], [n[1]], [9, 13, 8]])
    dims = [p[1] for p in parts]
    sl = lambda a, off, d: a[off[2]:off[2] + d[2], off[1]:off[1] + d[1], off[0]:off[0] + d[0]]
    inputs = [(np.ascontiguousarray(sl(coords, o, d)), np.ascontiguousarray(sl(q, o, d))) for o, d in parts]
    with _batch(dims, inputs, opts=opts) as bt:
        bt.set_halo_maps(B.halo_maps_decomposed(M, parts))
        bt.RungeKutta(steps, per_block=per_block)
        got = [bt.Q(k) for k in range(len(dims))]
    for (o, d), g in zip(parts, got):
        assert np.array_equal(g, sl(want, o, d)), max(per_field_rel_l2(g, sl(want, o, d)))


def test_mixed_batch_within_bar_of_fp64():
    inputs = _inputs(DIMS)
    steps = 20
    with _batch(DIMS, inputs, precision="mixed") as bt:
        bt.halo_periodic()
        bt.RungeKutta(steps)
        got = [bt.Q(k) for k in range(len(DIMS))]
    for d, (coords, q), g in zip(DIMS, inputs, got):
        want = _single(d, coords, q, steps)
        err = per_field_rel_l2(g, want)
        assert max(err) <= 1e-5, err


def test_donor_map_persistent_equals_per_block():
    from chimera_comp_les_b200 import batch as B
    dims = DIMS + [(18, 16, 22)]
    inputs = _inputs(dims, seed0=3)
    maps = B.halo_maps_donor(dims, [2, 3, 1, 0])
    res = []
    for per_block in (False, True):
        with _batch(dims, inputs) as bt:
            bt.set_halo_maps(maps)
            bt.RungeKutta(4, per_block=per_block)  # raises on NaN / rho or p <= 0
            res.append([bt.Q(k) for k in range(len(dims))])
    for a, b in zip(*res):
        assert np.isfinite(a).all()
        assert np.array_equal(a, b)


def test_autotune_keeps_state_and_results():
    inputs = _inputs(DIMS)
    with _batch(DIMS, inputs) as bt:
        bt.halo_periodic()
        bt.RungeKutta(1)
        before = [bt.Q(k) for k in range(len(DIMS))]
        kc, ms = bt.autotune()
        assert kc in (6, 8, 12, 16, 24, 32, 48) and ms > 0
        after = [bt.Q(k) for k in range(len(DIMS))]
        for x, y in zip(before, after):
            assert np.array_equal(x, y)
        bt.RungeKutta(2)
        got = [bt.Q(k) for k in range(len(DIMS))]
    for d, (coords, q), g in zip(DIMS, inputs, got):
        assert np.array_equal(g, _single(d, coords, q, 3))


def test_halo_map_errors():
    from chimera_comp_les_b200._lib import CB_E_ARG, CB_E_STATE, ChimeraError
    from chimera_comp_les_b200 import batch as B
    inputs = _inputs(DIMS)
    with _batch(DIMS, inputs) as bt:
        with pytest.raises(ChimeraError) as e:
            bt.RungeKutta(1)  # no halo map yet
        assert e.value.code == CB_E_STATE
        st, wr = B.halo_maps_self_periodic(DIMS)
        bad = st.copy()
        bad[0, 1:4] = (3, 3, 3)  # interior destination
        with pytest.raises(ChimeraError) as e:
            bt.set_halo_map(B.HALO_STAGE, bad)
        assert e.value.code == CB_E_ARG
        bad = wr.copy()
        bad[0, 5:8] = bad[1, 1:4]  # wrap source that is also a destination
        with pytest.raises(ChimeraError) as e:
            bt.set_halo_map(B.HALO_WRAP, bad)
        assert e.value.code == CB_E_ARG


def test_batch_cfl_dt_is_the_max_over_blocks():
    """cb_batch_cfl_dt over three blocks equals the largest single-block
    cb_cfl_dt radius, before and after steps (the current state buffer)."""
    from chimera_comp_les_b200 import Block
    inputs = _inputs(DIMS, seed0=5)
    with _batch(DIMS, inputs) as bt:
        bt.halo_periodic()
        for steps in (0, 2):
            if steps:
                bt.RungeKutta(steps)
            dt, lam = bt.cfl_dt(0.4)
            lams = []
            for k, (d, (coords, _)) in enumerate(zip(DIMS, inputs)):
                with Block(*d, **OPTS) as blk:
                    blk.FormMetrics(coords)
                    blk.SetInitialCondition(bt.Q(k))
                    lams.append(blk.cfl_dt(0.4)[1])
            assert lam == max(lams) and lam > 0
            assert dt == 0.4 / lam


def test_sensor_refused_with_a_cross_process_exchange():
    """The sensor's ghost layers cross blocks through the local wrap map only:
    a batch with the sensor refuses exchange lists with CB_E_UNSUPPORTED."""
    import torch
    from chimera_comp_les_b200._lib import CB_E_UNSUPPORTED, ChimeraError
    from chimera_comp_les_b200 import batch as B
    d = (14, 12, 11)
    inputs = _inputs([d], seed0=5)
    buf = torch.zeros(5, dtype=torch.float64, device="cuda:0")
    with _batch([d], inputs, opts=dict(OPTS, calc_sigma=1)) as bt:
        with pytest.raises(ChimeraError) as e:
            bt.set_exchange(B.HALO_STAGE, np.array([[0, 1, 1, 1, 0]]), buf.data_ptr(), np.zeros((0, 4)), 0)
        assert e.value.code == CB_E_UNSUPPORTED
