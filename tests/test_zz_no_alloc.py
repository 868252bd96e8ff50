"""cb_rhs_noalloc: formRHS for callers that cannot allocate device memory.

Such callers (a solver inside another framework's memory pool, a host that
forbids device allocation after start-up) pass device arrays they own and get
the RHS in a device array they own; the entry point's scratch is a file-scope
device array shared by all calls.  This test checks it against the existing
entry point (cb_rhs through a context) on successive calls with different
states, grids and options (with and without an eddy-viscosity array), so a
stale scratch value from an earlier call would show in a later one.  The
test allocates its own device buffers with torch -- that is the caller's
memory, not the entry point's.
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from chimera_comp_les_b200 import _lib
from chimera_comp_les_b200 import workloads as W

from _common import RTOL_L2, gpu_block, per_field_rel_l2

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def _existing_rhs(cfg, coords, q, nv):
    with gpu_block(cfg) as b:
        b.FormMetrics(coords)
        b.set_nvert(nv)
        b.SetInitialCondition(q)
        nut = None
        if cfg.les and not cfg.inviscid:
            b.CalcUCat()
            b.Compute_eddy_viscosity_LES()
            nut = b.nu_t()
        return b.formRHS(0), nut


def _cfg_struct(block_cfg):
    return C.byref(block_cfg)


# calls made in this order on the shared scratch: LES with a mask and a
# caller-supplied eddy viscosity, then a different grid (another padded plane
# size over the same array), then molecular viscosity only and an inviscid
# run, both without an eddy-viscosity array (d_nut NULL: zero)
CALLS = [
    dict(n=(30, 17, 22), seed=21, les=1, inviscid=0, mask=True, nut=True),
    dict(n=(33, 20, 18), seed=22, les=1, inviscid=0, mask=True, nut=True),
    dict(n=(26, 22, 19), seed=23, les=0, inviscid=0, mask=False, nut=False),
    dict(n=(24, 18, 20), seed=24, les=0, inviscid=1, mask=True, nut=False),
]


def test_noalloc_rhs_matches_existing_entry_point_on_successive_calls():
    import torch

    lib = _lib.load()
    for call, c in enumerate(CALLS):
        n = c["n"]
        coords = W.periodic_grid(n, 2 * np.pi, amp=0.05)
        shape = coords.shape[:3]
        cfg = O.Config(mx=n[0] + 2, my=n[1] + 2, mz=n[2] + 2, les=c["les"], inviscid=c["inviscid"], fluxorder=2,
                       ren=1600., ma=0.1, pr=0.71, dt=1e-3)
        nv = np.zeros(shape)
        if c["mask"]:
            nv[8:11, 7:10, 12:16] = 3.0
            nv[7:12, 6:11, 11:17][nv[7:12, 6:11, 11:17] == 0] = 1.0
        with gpu_block(cfg) as b:
            ccfg = b.cfg  # the C-ABI config struct of an equivalent context
        q = W.random_smooth_state(shape, seed=c["seed"])
        ref, nut = _existing_rhs(cfg, coords, q, nv)
        assert (nut is not None) == c["nut"]
        d_coor, d_nv, d_q = _dev(coords), _dev(nv), _dev(q)
        d_nut = _dev(nut) if c["nut"] else None
        d_rhs = torch.full(shape + (5,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = lib.cb_rhs_noalloc(C.byref(ccfg), d_coor.data_ptr(), d_q.data_ptr(), d_nv.data_ptr(),
                                d_nut.data_ptr() if d_nut is not None else None, d_rhs.data_ptr(), None)
        assert rc == 0, f"call {call}: status {rc}"
        torch.cuda.synchronize()
        got = d_rhs.cpu().numpy()
        errs = per_field_rel_l2(got, ref)
        assert max(errs) <= RTOL_L2, (call, errs)


def test_noalloc_rejects_grid_above_limit():
    import torch

    lib = _lib.load()
    m = 70  # (70+4 -> 80) * 74 * 74 padded nodes > CB_NOALLOC_MAX_PLANE
    ccfg = _lib.CbConfig()
    lib.cb_config_default(C.byref(ccfg), m, m, m)
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = dummy.data_ptr()
    assert lib.cb_rhs_noalloc(C.byref(ccfg), p, p, p, p, p, None) == _lib.CB_E_ARG
