"""Batched blocks with their own face codes (cb_batch_set_bctype).

The reference reads one bcs.dat line per block (init.c:556-559) and ends
every RK stage of every block with that block's FormBCS (solvers.c:246-273,
rhs.c:477-1227).  A batch that mixes such blocks with interface blocks (fed
by the self-periodic halo maps) must advance every block exactly as a
single-block context with the same codes: FP64 bit for bit, the mixed form
within 1e-7 of its own single-block runs (a chunk's first k-face may round
differently in the last bit when launch shapes differ).  One coded block is
also held to the oracle restatement, which is bit-exact against the
reference's FormBCS (tests/test_oracle_vs_reference.py).
"""
import numpy as np
import pytest

import oracle as O
from _common import RTOL_L2, oracle_run, per_field_rel_l2
from chimera_comp_les_b200 import workloads as W

pytestmark = pytest.mark.gpu

BASE = dict(inviscid=0, eno_order=2, central=2, ren=250.0, ma=0.3, pr=0.71, gamma=1.4, dt=2e-3)
DIMS = [(37, 19, 25), (26, 22, 20), (22, 30, 18), (34, 18, 24)]
# per block: its face codes, or None for an interface block of the halo maps
BCT = [(3, 3, 1, 1, 45, 44), None, (7, 7, 1, 1, 7, 7), (1, 1, 1, 1, 44, 45)]
CASES = [
    # WENO3 blend with the isothermal walls
    ("les_weno3_iso", dict(les=1, fluxorder=3, isothermal=1, s_x=0.4, s_y=0.7, s_z=0.9)),
    # MUSCL at sigma 0: without coded blocks the batch would launch the
    # periodic-only (PLAIN) variants, which fold the boundary branches away
    ("les_muscl_sigma0", dict(les=1, fluxorder=2, s_x=0.0, s_y=0.0, s_z=0.0)),
    ("muscl_roe", dict(les=0, fluxorder=2, flux="roe")),
    # the shock sensor: a coded block fills its planes' ghosts itself
    ("sensor", dict(les=1, fluxorder=3, calc_sigma=1, s_x=0.5, s_y=0.6, s_z=0.7, s_x_min=0.05, sigma_thrsh=1e-4)),
    # the dynamic model on a coded block's own arrays
    ("dynamic", dict(les=2, fluxorder=3, max_cs=0.1, s_x=0.4, s_y=0.7, s_z=0.9)),
]


def _inputs():
    out = []
    for b, (d, bc) in enumerate(zip(DIMS, BCT)):
        n = (d[0] - 2, d[1] - 2, d[2] - 2)
        coords = W.periodic_grid(n, 2 * np.pi, amp=0.04)
        q = W.random_smooth_state(coords.shape[:3], seed=20 + b, periodic=bc is None)
        out.append((coords, q))
    return out


def _single(d, bc, coords, q, steps, precision, opts):
    from chimera_comp_les_b200 import Block
    with Block(*d, bctype=bc or (7,) * 6, precision=precision, **opts) as blk:
        blk.FormMetrics(coords)
        blk.SetInitialCondition(q)
        blk.RungeKutta(steps)
        return blk.Q()


def _batch(inputs, precision, opts):
    from chimera_comp_les_b200.batch import Batch
    bt = Batch(DIMS, precision=precision, **opts)
    for k, bc in enumerate(BCT):
        if bc is not None:
            bt.set_bctype(k, bc)
    for k, (coords, q) in enumerate(inputs):
        bt.FormMetrics(k, coords)
        bt.SetInitialCondition(k, q)
    bt.halo_periodic()  # the interface block only: coded blocks wrap themselves
    return bt


@pytest.mark.parametrize("per_block", [False, True])
@pytest.mark.parametrize("name,over", CASES, ids=[c[0] for c in CASES])
def test_coded_blocks_equal_single_blocks(name, over, per_block):
    opts = dict(BASE, **over)
    inputs = _inputs()
    steps = 2
    for prec in ("fp64", "mixed"):
        with _batch(inputs, prec, opts) as bt:
            bt.RungeKutta(steps, per_block=per_block)
            got = [bt.Q(k) for k in range(len(DIMS))]
        for d, bc, (coords, q), g in zip(DIMS, BCT, inputs, got):
            want = _single(d, bc, coords, q, steps, prec, opts)
            assert np.isfinite(g).all()
            if prec == "fp64":
                assert np.array_equal(g, want), (bc, max(per_field_rel_l2(g, want)))
            else:
                assert max(per_field_rel_l2(g, want)) <= 1e-7, bc


def test_coded_block_matches_oracle():
    """Block 0 (slip walls, no-slip walls, inflow/outflow 45/44) after 3 steps
    against the CPU restatement of the reference."""
    opts = dict(BASE, les=1, fluxorder=3, isothermal=1, s_x=0.4, s_y=0.7, s_z=0.9)
    inputs = _inputs()
    d = DIMS[0]
    cfg = O.Config(mx=d[0], my=d[1], mz=d[2], bctype=BCT[0], **opts)
    coords, q = inputs[0]
    want = oracle_run(cfg, coords, q, np.zeros(q.shape[:3]), steps=3)["q_steps"]
    with _batch(inputs, "fp64", opts) as bt:
        bt.RungeKutta(3)
        got = bt.Q(0)
    assert max(per_field_rel_l2(got, want)) <= RTOL_L2


def test_all_coded_batch_needs_no_halo_map():
    """A batch whose every block has face codes steps without halo maps, as
    the reference's independent blocks do."""
    from chimera_comp_les_b200.batch import Batch
    opts = dict(BASE, les=1, fluxorder=3, s_x=0.4, s_y=0.7, s_z=0.9)
    dims, bcs = [DIMS[0], DIMS[3]], [BCT[0], BCT[3]]
    inputs = [_inputs()[0], _inputs()[3]]
    with Batch(dims, **opts) as bt:
        for k, (bc, (coords, q)) in enumerate(zip(bcs, inputs)):
            bt.set_bctype(k, bc)
            bt.FormMetrics(k, coords)
            bt.SetInitialCondition(k, q)
        bt.RungeKutta(2)
        got = [bt.Q(k) for k in range(2)]
    for d, bc, (coords, q), g in zip(dims, bcs, inputs, got):
        assert np.array_equal(g, _single(d, bc, coords, q, 2, "fp64", opts))


def test_face_code_errors():
    import torch
    from chimera_comp_les_b200._lib import CB_E_ARG, CB_E_STATE, CB_E_UNSUPPORTED, ChimeraError
    from chimera_comp_les_b200 import batch as B
    opts = dict(BASE, les=1, fluxorder=3)
    inputs = _inputs()
    with _batch(inputs, "fp64", opts) as bt:
        # block 1 is an interface block holding halo-map destinations
        with pytest.raises(ChimeraError) as e:
            bt.set_bctype(1, (3, 3, 1, 1, 45, 44))
        assert e.value.code == CB_E_ARG
        with pytest.raises(ChimeraError) as e:
            bt.set_bctype(0, (7, 3, 1, 1, 45, 44))
        assert e.value.code == CB_E_UNSUPPORTED
        # the inflow codes 52 / 47 keep the coordinates of the grid upload
        with pytest.raises(ChimeraError) as e:
            bt.set_bctype(0, (3, 3, 1, 1, 52, 44))
        assert e.value.code == CB_E_STATE
        # a halo map may not write into a coded block
        st, _ = B.halo_maps_self_periodic(DIMS)
        with pytest.raises(ChimeraError) as e:
            bt.set_halo_map(B.HALO_STAGE, st[st[:, 0] == 0])
        assert e.value.code == CB_E_ARG
        # nor does a batch with coded blocks take a cross-process exchange
        buf = torch.zeros(5, dtype=torch.float64, device="cuda:0")
        with pytest.raises(ChimeraError) as e:
            bt.set_exchange(B.HALO_STAGE, np.array([[1, 1, 1, 1, 0]]), buf.data_ptr(), np.zeros((0, 4)), 0)
        assert e.value.code == CB_E_UNSUPPORTED


@pytest.mark.parametrize("les,ti0", [(0, 1), (1, 6)])
def test_inflow_codes_52_47_on_coded_blocks(les, ti0):
    """The k-lo inflow codes that read the node coordinates (52: the
    characteristic cos^2 inlet, rhs.c:854-874; 47: the power-law inlet with
    perturbations travelling in x and time, rhs.c:904-950, its step index from
    cb_batch_set_time_index) on two coded blocks beside an interface block,
    3 steps, bit for bit against single-block contexts."""
    from chimera_comp_les_b200 import Block
    from chimera_comp_les_b200.batch import Batch
    dims = [(37, 19, 25), (26, 22, 20), (34, 18, 24)]
    bcs = [(7, 7, 3, 3, 52, 44), None, (7, 7, 3, 3, 47, 45)]
    opts = dict(BASE, les=les, fluxorder=3, s_x=0.4 if les else 1.0, s_y=0.7, s_z=0.9, ren=250.)
    inputs = []
    for b, (d, bc) in enumerate(zip(dims, bcs)):
        coords = W.periodic_grid((d[0] - 2, d[1] - 2, d[2] - 2), 2 * np.pi, amp=0.04)
        if bc is not None:
            coords[..., 1] = 1.5 * coords[..., 1] + 1.0  # y on both sides of 47's y = 8
        inputs.append((coords, W.random_smooth_state(coords.shape[:3], seed=40 + b, periodic=bc is None)))
    with Batch(dims, **opts) as bt:
        for k, bc in enumerate(bcs):
            if bc is not None:
                bt.set_bctype(k, bc)
        for k, (coords, q) in enumerate(inputs):
            bt.FormMetrics(k, coords)
            bt.SetInitialCondition(k, q)
        bt.halo_periodic()
        bt.set_time_index(ti0 - 1)
        bt.RungeKutta(3)
        got = [bt.Q(k) for k in range(len(dims))]
    for d, bc, (coords, q), g in zip(dims, bcs, inputs, got):
        with Block(*d, bctype=bc or (7,) * 6, **opts) as blk:
            blk.FormMetrics(coords)
            blk.SetInitialCondition(q)
            blk.set_time_index(ti0 - 1)
            blk.RungeKutta(3)
            want = blk.Q()
        assert np.isfinite(g).all()
        assert np.array_equal(g, want), (bc, max(per_field_rel_l2(g, want)))
