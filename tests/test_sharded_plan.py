"""Multi-process halo exchange on the CPU: exchange plans and the
torch.distributed transport (gloo, world size 2 and 3).

Each process holds some sub-blocks of a decomposed periodic box as numpy
arrays, applies its local halo entries, packs what its peers need, exchanges
through ``DistTransport.exchange_buffers`` and unpacks; every block must then
hold exactly what the undivided box's rule (a scalar restatement of FormBCS,
rhs.c:1107-1227) gives, as when all blocks live in one process.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from chimera_comp_les_b200 import batch as B
from chimera_comp_les_b200 import sharded as S

from test_batch_maps import block_slice, global_stage, padded

CUTS = ([5, 6], [7], [4, 5, 6, 4])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _wrap_fill(M, g):
    w = lambda x, m: x + m if x < 0 else (x - m if x >= m else x)
    out = g.copy()
    for k in range(-2, M[2] + 2):
        for j in range(-2, M[1] + 2):
            for i in range(-2, M[0] + 2):
                out[k + 2, j + 2, i + 2] = g[w(k, M[2]) + 2, w(j, M[1]) + 2, w(i, M[0]) + 2]
    return out


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        M = tuple(sum(c) + 2 for c in CUTS)
        parts = B.decompose(M, CUTS)
        stage_map, wrap_map = B.halo_maps_decomposed(M, parts)
        rob = S.slab_ranks(len(parts), world)
        plan = S.exchange_plan(stage_map, wrap_map, rob, rank)
        tr = S.DistTransport()
        rng = np.random.default_rng(3)  # the same global fields in every process
        qin = [padded(M, rng) for _ in range(5)]
        qout = [padded(M, rng) for _ in range(5)]
        # ---- stage map: local entries, pack, exchange, unpack
        ins = {b: [block_slice(a, *parts[b]) for a in qin] for b in plan.blocks}
        outs = {}
        for b in plan.blocks:
            off, d = parts[b]
            fl = []
            for a in qout:
                o = block_slice(a, off, d)
                m = np.ones_like(o, dtype=bool)
                m[3:d[2] + 1, 3:d[1] + 1, 3:d[0] + 1] = False
                o[m] = np.nan  # not written by the stage: never a source
                fl.append(o)
            outs[b] = fl
        res = {b: [o.copy() for o in outs[b]] for b in plan.blocks}
        at = lambda a, i, j, k: a[k + 2, j + 2, i + 2]
        for r in plan.stage.local:
            sb, db = plan.blocks[r[4]], plan.blocks[r[0]]
            for f in range(5):
                src = ins[sb][f] if r[8] else outs[sb][f]
                res[db][f][r[3] + 2, r[2] + 2, r[1] + 2] = at(src, r[5], r[6], r[7])
        send = torch.zeros(len(plan.stage.send) * 5, dtype=torch.float64)
        for e, r in enumerate(plan.stage.send):
            sb = plan.blocks[r[0]]
            for f in range(5):
                send[e * 5 + f] = float(at(ins[sb][f] if r[4] else outs[sb][f], r[1], r[2], r[3]))
        recv = torch.zeros(len(plan.stage.recv) * 5, dtype=torch.float64)
        tr.exchange_buffers(plan, plan.stage, send, recv, 5)
        for e, r in enumerate(plan.stage.recv):
            db = plan.blocks[r[0]]
            for f in range(5):
                res[db][f][r[3] + 2, r[2] + 2, r[1] + 2] = float(recv[e * 5 + f])
        want = [global_stage(M, qin[f], qout[f]) for f in range(5)]
        ok_stage = all(np.array_equal(res[b][f], block_slice(want[f], *parts[b])) for b in plan.blocks for f in range(5))
        # ---- wrap map (1 field, the eddy-viscosity case)
        g = qin[0]
        wantw = _wrap_fill(M, g)
        arr = {}
        for b in plan.blocks:
            off, d = parts[b]
            a = block_slice(wantw, off, d)
            for k in range(-2, d[2] + 2):
                for j in range(-2, d[1] + 2):
                    for i in range(-2, d[0] + 2):
                        own = 0 <= i < d[0] and 0 <= j < d[1] and 0 <= k < d[2]
                        gi, gj, gk = i + off[0], j + off[1], k + off[2]
                        gint = 1 <= gi <= M[0] - 2 and 1 <= gj <= M[1] - 2 and 1 <= gk <= M[2] - 2
                        inter = 1 <= i <= d[0] - 2 and 1 <= j <= d[1] - 2 and 1 <= k <= d[2] - 2
                        if not own or (not inter and gint):
                            a[k + 2, j + 2, i + 2] = np.nan
            arr[b] = a
        sendw = torch.tensor([float(at(arr[plan.blocks[r[0]]], r[1], r[2], r[3])) for r in plan.wrap.send],
                             dtype=torch.float64) if len(plan.wrap.send) else torch.zeros(1, dtype=torch.float64)
        for r in plan.wrap.local:  # sources are never destinations: order does not matter
            arr[plan.blocks[r[0]]][r[3] + 2, r[2] + 2, r[1] + 2] = at(arr[plan.blocks[r[4]]], r[5], r[6], r[7])
        recvw = torch.zeros(max(len(plan.wrap.recv), 1), dtype=torch.float64)
        tr.exchange_buffers(plan, plan.wrap, sendw, recvw, 1)
        for e, r in enumerate(plan.wrap.recv):
            arr[plan.blocks[r[0]]][r[3] + 2, r[2] + 2, r[1] + 2] = float(recvw[e])
        ok_wrap = all(np.array_equal(arr[b], block_slice(wantw, *parts[b])) for b in plan.blocks)
        q.put((rank, ok_stage, ok_wrap, len(plan.stage.send), len(plan.stage.recv), plan.peers))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_exchange_reproduces_undivided_box(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=240) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs)
    for rank, ok_stage, ok_wrap, ns, nr, peers in res:
        assert ok_stage and ok_wrap, rank
        assert ns > 0 and nr > 0 and peers


def test_plan_counts_are_symmetric():
    M = tuple(sum(c) + 2 for c in CUTS)
    parts = B.decompose(M, CUTS)
    st, wr = B.halo_maps_decomposed(M, parts)
    world = 3
    rob = S.slab_ranks(len(parts), world)
    plans = [S.exchange_plan(st, wr, rob, r) for r in range(world)]
    for a in plans:
        for b in plans:
            if a.rank == b.rank:
                continue
            for kind in ("stage", "wrap"):
                assert getattr(a, kind).send_counts.get(b.rank, 0) == getattr(b, kind).recv_counts.get(a.rank, 0)
    # every destination of the global map lands exactly once: locally or received
    total = sum(len(p.stage.local) + len(p.stage.recv) for p in plans)
    assert total == len(st)


class _StubBatch:
    """Stands in for a Batch: its own largest spectral radius."""

    def __init__(self, lam):
        self.lam = lam

    def cfl_dt(self, cfl):
        return cfl / self.lam, self.lam


class _StubShard:
    def __init__(self, lam):
        self.batch = _StubBatch(lam)


def _cfl_worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # rank r holds two shards; the global largest radius sits on the last rank
        shards = [_StubShard(1.0 + rank), _StubShard(0.5 + 2.0 * rank)]
        q.put((rank,) + S.cfl_dt(shards, 0.4))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_cfl_dt_takes_the_global_max(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_cfl_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=240) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs)
    lam = max(1.0 + (world - 1), 0.5 + 2.0 * (world - 1))
    for rank, dt, got in res:
        assert got == lam and dt == 0.4 / lam, rank


def test_cfl_dt_without_a_process_group():
    dt, lam = S.cfl_dt([_StubShard(2.0), _StubShard(3.0)], 0.3)
    assert lam == 3.0 and dt == 0.3 / 3.0
