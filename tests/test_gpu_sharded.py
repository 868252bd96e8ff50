"""The cross-process exchange path on one GPU: the sub-blocks of a periodic
box split across two "processes", each its own Batch, exchanging through the
same phase API (pack, transfer, unpack) that NCCL ranks use; the transfer is a
device copy here (LocalTransport).  The result must equal the undivided box
bit-for-bit (FP64), with the 2-point central flux (the reference's 4-point
flux is switched off on block faces, rhs.c:3483-3547)."""
import math

import numpy as np
import pytest

from _common import per_field_rel_l2

pytestmark = pytest.mark.gpu

OPTS = dict(les=1, inviscid=0, fluxorder=3, eno_order=2, central=1, ren=1600.0, ma=0.1, pr=0.71, gamma=1.4, dt=2e-3)


def _k_uniform_grid(n):
    from chimera_comp_les_b200 import workloads as W
    length = (2 * math.pi, 2 * math.pi, n[2] * 0.25)
    g = W.periodic_grid(n, length, 0.0)
    sx = 2 * math.pi * g[..., 0] / length[0]
    sy = 2 * math.pi * g[..., 1] / length[1]
    g[..., 0] += 0.04 * np.sin(sy)
    g[..., 1] += 0.03 * np.sin(sx)
    return np.ascontiguousarray(g)


@pytest.mark.parametrize("world,per_block", [(2, False), (3, True)])
def test_sharded_box_equals_undivided(world, per_block):
    import torch

    from chimera_comp_les_b200 import Block
    from chimera_comp_les_b200 import batch as B
    from chimera_comp_les_b200 import sharded as S
    from chimera_comp_les_b200 import workloads as W
    n = (22, 18, 30)
    M = (n[0] + 2, n[1] + 2, n[2] + 2)
    coords = _k_uniform_grid(n)
    q = W.isotropic_turbulence(n, 17, k_peak=3.0, mach_t=0.3)
    steps = 3
    with Block(*M, **OPTS) as blk:
        blk.FormMetrics(coords)
        blk.SetInitialCondition(q)
        blk.RungeKutta(steps)
        want = blk.Q()
    parts = B.decompose(M, [[n[0]], [n[1]], [9, 13, 8]])
    st, wr = B.halo_maps_decomposed(M, parts)
    rob = S.slab_ranks(len(parts), world)
    sl = lambda a, off, d: a[off[2]:off[2] + d[2], off[1]:off[1] + d[1], off[0]:off[0] + d[0]]
    shards = []
    for r in range(world):
        plan = S.exchange_plan(st, wr, rob, r)
        bt = B.Batch([parts[b][1] for b in plan.blocks], **OPTS)
        for k, b in enumerate(plan.blocks):
            o, d = parts[b]
            bt.FormMetrics(k, np.ascontiguousarray(sl(coords, o, d)))
            bt.SetInitialCondition(k, np.ascontiguousarray(sl(q, o, d)))
        shards.append(S.Shard(bt, plan, torch.device("cuda:0")))
    tr = S.LocalTransport()
    S.fill_ghosts_all(shards, tr)
    S.step_all(shards, tr, steps, per_block=per_block)
    for sh in shards:
        sh.batch.sync()
        for k, b in enumerate(sh.plan.blocks):
            o, d = parts[b]
            got = sh.batch.Q(k)
            assert np.array_equal(got, sl(want, o, d)), (b, max(per_field_rel_l2(got, sl(want, o, d))))
    for sh in shards:
        sh.batch.close()


def test_exchange_batch_refuses_graph_step():
    import torch

    from chimera_comp_les_b200 import batch as B
    from chimera_comp_les_b200 import sharded as S
    from chimera_comp_les_b200 import workloads as W
    from chimera_comp_les_b200._lib import CB_E_STATE, ChimeraError
    n = (12, 10, 16)
    M = (n[0] + 2, n[1] + 2, n[2] + 2)
    parts = B.decompose(M, [[n[0]], [n[1]], [8, 8]])
    st, wr = B.halo_maps_decomposed(M, parts)
    plan = S.exchange_plan(st, wr, [0, 1], 0)
    coords = _k_uniform_grid(n)
    q = W.isotropic_turbulence(n, 5, k_peak=2.0, mach_t=0.2)
    o, d = parts[0]
    with B.Batch([d], **OPTS) as bt:
        bt.FormMetrics(0, np.ascontiguousarray(coords[o[2]:o[2] + d[2]]))
        bt.SetInitialCondition(0, np.ascontiguousarray(q[o[2]:o[2] + d[2]]))
        sh = S.Shard(bt, plan, torch.device("cuda:0"))
        with pytest.raises(ChimeraError) as e:
            bt.RungeKutta(1)
        assert e.value.code == CB_E_STATE
        del sh
