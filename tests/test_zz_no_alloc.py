"""cb_rhs_noalloc: formRHS for callers that cannot allocate device memory.

Such callers (a solver inside another framework's memory pool, a host that
forbids device allocation after start-up) pass device arrays they own and get
the RHS in a device array they own; the entry point's scratch is a file-scope
device array shared by all calls.  This test checks it against the existing
entry point (cb_rhs through a context) on two calls in a row with different
states, so a stale scratch value from the first call would show in the
second.  The test allocates its own device buffers with torch -- that is the
caller's memory, not the entry point's.
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


def test_noalloc_rhs_matches_existing_entry_point_twice():
    import torch

    lib = _lib.load()
    n = (30, 17, 22)
    coords = W.periodic_grid(n, 2 * np.pi, amp=0.05)
    shape = coords.shape[:3]
    cfg = O.Config(mx=n[0] + 2, my=n[1] + 2, mz=n[2] + 2, les=1, inviscid=0, fluxorder=2, ren=1600., ma=0.1,
                   pr=0.71, dt=1e-3)
    nv = np.zeros(shape)
    nv[8:11, 7:10, 12:16] = 3.0
    nv[7:12, 6:11, 11:17][nv[7:12, 6:11, 11:17] == 0] = 1.0
    with gpu_block(cfg) as b:
        ccfg = b.cfg  # the C-ABI config struct of an equivalent context
    d_coor, d_nv = _dev(coords), _dev(nv)
    for call, seed in enumerate((21, 22)):
        q = W.random_smooth_state(shape, seed=seed)
        ref, nut = _existing_rhs(cfg, coords, q, nv)
        d_q, d_nut = _dev(q), _dev(nut)
        d_rhs = torch.full(shape + (5,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = lib.cb_rhs_noalloc(C.byref(ccfg), d_coor.data_ptr(), d_q.data_ptr(), d_nv.data_ptr(),
                                d_nut.data_ptr(), d_rhs.data_ptr(), None)
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
