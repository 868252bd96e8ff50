"""One domain across several processes (one per GPU): halo exchange plans and
the per-stage exchange.

The reference decomposes each block into a 3-D box per MPI rank and refreshes
the two-node DMDA ghosts inside DMGlobalToLocal (init.c:156, 206-218), with
the periodic FormBCS copy in between (rhs.c:1107-1227).  Here a domain is a
set of blocks (``batch.decompose`` of a periodic box, or any multi-block set)
with GLOBAL halo maps (``batch.halo_maps_*``); every process holds some of the
blocks in a ``Batch`` and exchanges, after each stage, exactly the halo
entries whose source block lives in another process:

  plan = exchange_plan(stage_map, wrap_map, rank_of_block, rank)
  sh = Shard(batch, plan, transport)       # transport: DistTransport / LocalTransport
  step_all([sh], transport, nsteps)

Per stage: the stage kernel and the local halo gather, a pack of the values
the peers need into one device buffer (entry-major), one grouped send/recv per
peer (NCCL over NVLink through ``torch.distributed``, on the batch's stream),
an unpack into the halo.  Entries are ordered by global map index on both
sides, so sender and receiver agree without exchanging metadata.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List, Sequence

import numpy as np

from ._lib import CB_PHASE_NUT, CB_PHASE_STAGE, CB_PHASE_STATE
from .batch import HALO_STAGE, HALO_WRAP


@dataclass
class KindPlan:
    """One map kind (stage or wrap) as seen by one process."""
    local: np.ndarray                                        # (n, 9) entries with local block ids
    send: np.ndarray                                         # (ns, 5) local src (block, i, j, k, from_stage_input)
    recv: np.ndarray                                         # (nr, 4) local dst (block, i, j, k)
    send_counts: Dict[int, int] = field(default_factory=dict)  # peer -> entries, in peer order
    recv_counts: Dict[int, int] = field(default_factory=dict)


@dataclass
class Plan:
    rank: int
    blocks: List[int]          # global ids of the blocks this process holds, in local order
    peers: List[int]           # other processes this one exchanges with, ascending
    stage: KindPlan
    wrap: KindPlan


def _split(m: np.ndarray, rank_of_block: np.ndarray, rank: int, local_id: np.ndarray) -> KindPlan:
    rd = rank_of_block[m[:, 0]]
    rs = rank_of_block[m[:, 4]]
    loc = m[(rd == rank) & (rs == rank)].copy()
    loc[:, 0] = local_id[loc[:, 0]]
    loc[:, 4] = local_id[loc[:, 4]]
    # receive: destination here, source elsewhere; ordered by (source rank, global index)
    ri = np.nonzero((rd == rank) & (rs != rank))[0]
    ri = ri[np.lexsort((ri, rs[ri]))]
    recv = m[ri][:, 0:4].copy()
    recv[:, 0] = local_id[recv[:, 0]]
    # send: source here, destination elsewhere; ordered by (destination rank, global index)
    si = np.nonzero((rs == rank) & (rd != rank))[0]
    si = si[np.lexsort((si, rd[si]))]
    send = m[si][:, 4:9].copy()
    send[:, 0] = local_id[send[:, 0]]
    rc = {int(p): int(c) for p, c in zip(*np.unique(rs[ri], return_counts=True))}
    sc = {int(p): int(c) for p, c in zip(*np.unique(rd[si], return_counts=True))}
    return KindPlan(np.ascontiguousarray(loc, dtype=np.int32), np.ascontiguousarray(send, dtype=np.int32),
                    np.ascontiguousarray(recv, dtype=np.int32), sc, rc)


def exchange_plan(stage_map: np.ndarray, wrap_map: np.ndarray, rank_of_block: Sequence[int], rank: int) -> Plan:
    """This process's share of global halo maps (global block ids)."""
    rob = np.asarray(rank_of_block, dtype=np.int64)
    blocks = [int(b) for b in np.nonzero(rob == rank)[0]]
    local_id = np.full(len(rob), -1, dtype=np.int64)
    local_id[blocks] = np.arange(len(blocks))
    st = _split(np.asarray(stage_map), rob, rank, local_id)
    wr = _split(np.asarray(wrap_map), rob, rank, local_id)
    peers = sorted(set(st.send_counts) | set(st.recv_counts) | set(wr.send_counts) | set(wr.recv_counts))
    return Plan(rank, blocks, peers, st, wr)


def slab_ranks(nparts: int, world: int) -> List[int]:
    """Contiguous slabs: part p of nparts to process p * world // nparts."""
    return [p * world // nparts for p in range(nparts)]


# -------------------------------------------------------------- transports --
def _chunks(counts: Dict[int, int], peers: Sequence[int], nf: int):
    off, out = 0, {}
    for p in peers:
        c = counts.get(p, 0)
        out[p] = (off * nf, (off + c) * nf)
        off += c
    return out


class DistTransport:
    """Grouped point-to-point send/recv through ``torch.distributed`` (NCCL on
    GPUs, gloo on CPU tensors).  Every process calls ``exchange`` for the same
    kinds in the same order; each pair posts its sends and receives in one
    ``batch_isend_irecv``."""

    def __init__(self, group=None):
        self.group = group

    def exchange_buffers(self, plan: Plan, kp: KindPlan, send, recv, nf: int):
        import torch.distributed as dist
        sc = _chunks(kp.send_counts, plan.peers, nf)
        rc = _chunks(kp.recv_counts, plan.peers, nf)
        ops = []
        for p in plan.peers:
            a, b = rc[p]
            if b > a:
                ops.append(dist.P2POp(dist.irecv, recv[a:b], p, group=self.group))
            a, b = sc[p]
            if b > a:
                ops.append(dist.P2POp(dist.isend, send[a:b], p, group=self.group))
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()

    def exchange(self, shards, kind: int, nf: int):
        import torch
        (sh,) = shards
        kp = sh.plan.stage if kind == HALO_STAGE else sh.plan.wrap
        send, recv = sh.buffers(kind)
        # order the transfer after this batch's packs and before its unpacks
        with torch.cuda.stream(torch.cuda.ExternalStream(sh.batch.stream, device=send.device)):
            self.exchange_buffers(sh.plan, kp, send, recv, nf)


class LocalTransport:
    """Several processes' shards held by ONE process on one GPU (each its own
    Batch): the transfer is a device copy of each sender's chunk into the
    receiver's buffer.  Used to test the exchange path without a second GPU."""

    def exchange(self, shards, kind: int, nf: int):
        import torch
        by_rank = {sh.plan.rank: sh for sh in shards}
        torch.cuda.synchronize()
        for sh in shards:
            kp_r = sh.plan.stage if kind == HALO_STAGE else sh.plan.wrap
            _, recv = sh.buffers(kind)
            rc = _chunks(kp_r.recv_counts, sh.plan.peers, nf)
            for p in sh.plan.peers:
                a, b = rc[p]
                if b == a:
                    continue
                src = by_rank[p]
                kp_s = src.plan.stage if kind == HALO_STAGE else src.plan.wrap
                send, _ = src.buffers(kind)
                sa, sb = _chunks(kp_s.send_counts, src.plan.peers, nf)[sh.plan.rank]
                assert sb - sa == b - a, "send and receive plans disagree"
                recv[a:b].copy_(send[sa:sb])
        torch.cuda.synchronize()


# ------------------------------------------------------------------- shard --
class Shard:
    """A Batch holding this process's blocks, with its exchange lists and
    device buffers (torch tensors, 5 doubles per entry)."""

    def __init__(self, batch, plan: Plan, device):
        import torch
        self.batch, self.plan = batch, plan
        batch.set_halo_map(HALO_STAGE, plan.stage.local)
        batch.set_halo_map(HALO_WRAP, plan.wrap.local)
        mk = lambda n: torch.zeros(max(n, 1) * 5, dtype=torch.float64, device=device)
        self._buf = {HALO_STAGE: (mk(len(plan.stage.send)), mk(len(plan.stage.recv))),
                     HALO_WRAP: (mk(len(plan.wrap.send)), mk(len(plan.wrap.recv)))}
        for kind, kp in ((HALO_STAGE, plan.stage), (HALO_WRAP, plan.wrap)):
            s, r = self._buf[kind]
            send = kp.send if kind == HALO_STAGE else kp.send[:, 0:4]
            batch.set_exchange(kind, send, s.data_ptr(), kp.recv, r.data_ptr())

    def buffers(self, kind: int):
        return self._buf[kind]


def reduce_max(x: float, group=None) -> float:
    """Max of one scalar over the processes of ``group`` (one all_reduce; NCCL
    on a CUDA tensor, gloo on a CPU one); x itself outside torch.distributed."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(x)
    on_gpu = dist.get_backend(group) == "nccl"
    dev = torch.device("cuda", torch.cuda.current_device()) if on_gpu else torch.device("cpu")
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def cfl_dt(shards, cfl: float, group=None):
    """CFL time step of the whole domain: the largest spectral radius of this
    process's shards (``Batch.cfl_dt``), then the max over processes.  Every
    process gets the same (dt, lambda_max).  No reference counterpart: the
    reference steps with the fixed -dt (init.c:94)."""
    lam = max(sh.batch.cfl_dt(cfl)[1] for sh in shards)
    lam = reduce_max(lam, group)
    return (cfl / lam if lam > 0 else 0.0), lam


def _run_phase(shards, transport, phase, stage, kind, nf, per_block):
    for sh in shards:
        sh.batch.phase(phase, stage, per_block)
    transport.exchange(shards, kind, nf)
    for sh in shards:
        sh.batch.phase_unpack(phase)


def fill_ghosts_all(shards, transport):
    """Once after the uploads: ghosts of the initial state from the owners."""
    _run_phase(shards, transport, CB_PHASE_STATE, 0, HALO_WRAP, 5, False)


def step_all(shards, transport, nsteps: int = 1, per_block: bool = False):
    """nsteps RK steps of every shard (all shards of this process together)."""
    cfg = shards[0].batch.cfg
    for _ in range(nsteps):
        if cfg.les and not cfg.inviscid:
            _run_phase(shards, transport, CB_PHASE_NUT, 0, HALO_WRAP, 1, per_block)
        for s in range(cfg.fluxorder):
            _run_phase(shards, transport, CB_PHASE_STAGE, s, HALO_STAGE, 5, per_block)
