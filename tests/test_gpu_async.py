"""Streaming host transfers (cb_upload_state_async / cb_download_state_async /
cb_join_transfers): a host that hands every step its input and takes every
step's result gets exactly what the blocking calls give, through several
rounds of the double-buffered staging."""
import math

import numpy as np
import pytest

from chimera_comp_les_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_async_transfers_equal_blocking_calls(precision):
    import torch

    from chimera_comp_les_b200 import Block
    n = (34, 20, 18)
    coords = W.periodic_grid(n, 2 * math.pi, amp=0.05)
    kw = dict(les=1, fluxorder=2, s_x=0.0, s_y=0.0, s_z=0.0, ren=1600.0, ma=0.1, pr=0.71, dt=1e-3, precision=precision)
    states = [W.tgv_state(coords, gamma=1.4, ma=0.1)]
    for s in range(4):
        q = states[0].copy()
        q[..., 4] *= 1.0 + 1e-3 * (s + 1)  # distinct inputs per round
        states.append(q)
    steps = [1, 2, 1, 3, 2]
    pinned = lambda a: torch.empty(a.shape, dtype=torch.float64, pin_memory=True).numpy()  # noqa: E731
    with Block(n[0] + 2, n[1] + 2, n[2] + 2, **kw) as b:
        b.FormMetrics(coords)
        want = []
        for q, k in zip(states, steps):
            b.SetInitialCondition(q)
            b.RungeKutta(k)
            want.append(b.Q())
    with Block(n[0] + 2, n[1] + 2, n[2] + 2, **kw) as b:
        b.FormMetrics(coords)
        ins = [pinned(q) for q in states]
        for h, q in zip(ins, states):
            h[...] = q
        outs = [pinned(q) for q in states]
        for h, o, k in zip(ins, outs, steps):
            b.upload_async(h)
            b.RungeKutta(k, sync=False)
            b.download_async(o)
        b.join_transfers()
        b.sync()
    for o, w in zip(outs, want):
        assert np.array_equal(o, w)
