"""CPU baseline of the RHS + RK stage path on the host cores.

TEST/BENCH INFRASTRUCTURE ONLY: called by bench.py's cpu_baseline leg and its
``--impl reference`` arm, never by the product.

The reference's own hot path (oracle/_ref, built from rhs.c, les.c,
metrics.c, solvers.c against the serial PETSc shim) runs as P independent
processes, one per core, each advancing its own k-slab of the workload as a
periodic box with its own ghost layers.  This is an upper bound of the
reference's MPI path: the halo exchange between ranks is not performed.
When the reference build is absent the C restatement (``kind = "port"``)
runs instead.
"""
from __future__ import annotations

import math
import multiprocessing as mp
import os
import time


def _slab_worker(args):
    kind, optimized, n, nz, steps, warmup, cfgkw, barrier = args
    import numpy as np

    import oracle as O
    from chimera_comp_les_b200 import workloads as W

    coords = W.periodic_grid((n, n, nz), (2 * math.pi, 2 * math.pi, 2 * math.pi * nz / n), amp=0.05)
    cfg = O.Config(mx=n + 2, my=n + 2, mz=nz + 2, **cfgkw)
    q = W.tgv_state(coords, gamma=cfg.gamma, ma=cfg.ma)
    nv = np.zeros(coords.shape[:3])
    if kind == "reference":
        ref = O.RefOracle(cfg, coords, optimized=optimized)
        ref.set_nvert(nv)
        ref.set_state(q)
        step = lambda k: ref.steps(k)  # noqa: E731
    else:
        ora = O.Oracle(cfg)
        met = ora.metrics(O.to_padded(cfg, coords))
        nvp = ora.fill_ghosts(O.to_padded(cfg, nv))
        st = ora.initial_state(q)
        step = lambda k: ora.steps(k, st, met, nvp)  # noqa: E731
    if warmup:
        step(warmup)
    if barrier is not None:
        barrier.wait()
    t0 = time.time()
    step(steps)
    t1 = time.time()
    return t0, t1, n * n * nz * steps * cfg.nstages


def available_kind() -> str:
    import oracle as O
    return "reference" if os.path.exists(O.REF_SO_O3) or os.path.isdir(O.REF_SRC_DIR) else "port"


def run(n: int, steps: int, warmup: int = 0, procs: int = 0, cfgkw=None, kind: str = "", optimized: bool = True,
        nz: int = 0):
    """Returns dict(value=cell-updates/s per stage over all processes, cores,
    kind, seconds, sample).  nz: interior planes of each process's slab
    (default n // procs, the workload cut into procs slabs)."""
    cfgkw = dict(cfgkw or {})
    kind = kind or available_kind()
    procs = procs or min(os.cpu_count() or 1, 64)
    nz = nz or max(2, n // procs)
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        barrier = mgr.Barrier(procs)
        with ctx.Pool(procs) as pool:
            res = pool.map(_slab_worker, [(kind, optimized, n, nz, steps, warmup, cfgkw, barrier)] * procs)
    t0 = min(r[0] for r in res)
    t1 = max(r[1] for r in res)
    cells = sum(r[2] for r in res)
    secs = t1 - t0
    return {
        "value": cells / secs,
        "cores": procs,
        "kind": kind,
        "seconds": secs,
        "sample": (f"{procs} processes x {steps} RK steps of a {n}x{n}x{nz}-interior periodic k-slab "
                   f"({('reference rhs.c/les.c/solvers.c via PETSc shim, ' + ('-O3' if optimized else '-O0 as shipped')) if kind == 'reference' else 'oracle C restatement'})"
                   f"; no inter-slab halo exchange (upper bound of the MPI path)"),
    }
