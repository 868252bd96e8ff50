"""Floating-point operations per cell-update of the RHS + RK stage path.

TEST/BENCH INFRASTRUCTURE ONLY: bench.py's compute roofline uses these counts;
the product never imports this module.

The restatement (oracle/src/cb_oracle.c) is run through its counting build
(oracle/count/cbo_count.hpp: every operation on a double bumps a counter of
its kind) on a small periodic box of the workload, and the counts are divided
by the interior nodes:

* ``rhs``  -- one formRHS (EqOfState of the ghosted state, every face flux
  once, the flux differences, MultAj) per interior node;
* ``stage`` -- one whole time step (eddy viscosity once, every stage's RHS,
  RK combination and boundary fill) per interior node and stage: the
  arithmetic of one cell-update.

``flops`` counts add/sub, mul, div and sqrt as one operation each (pow and
other transcendentals counted apart); comparisons and fabs are listed but not
counted as flops.
"""
from __future__ import annotations

import numpy as np

from . import Config, Oracle, to_padded

FLOP_KINDS = ("add", "mul", "div", "sqrt")


def _flops(c: dict) -> int:
    return sum(c[k] for k in FLOP_KINDS)


def count_per_cell(cfgkw: dict, coords: np.ndarray, q: np.ndarray) -> dict:
    """Counts per interior node for the options cfgkw on the grid coords
    (natural (mz,my,mx,3)) and state q (natural (mz,my,mx,5))."""
    mz, my, mx = coords.shape[:3]
    cfg = Config(mx=mx, my=my, mz=mz, **cfgkw)
    ora = Oracle(cfg, counting=True)
    met = ora.metrics(to_padded(cfg, coords))
    nvp = ora.fill_ghosts(to_padded(cfg, np.zeros(coords.shape[:3])))
    interior = (mx - 2) * (my - 2) * (mz - 2)

    st = ora.initial_state(q)
    nut = ora.zeros(1)
    sig = ora.sigma(st["q"]) if cfg.les else None
    ora.count_reset()
    ora.rhs(st["q"], met, nvp, nut, sig)
    rhs = ora.count_read()

    st = ora.initial_state(q)
    ora.count_reset()
    ora.steps(1, st, met, nvp)
    step = ora.count_read()
    stages = cfg.nstages

    per = lambda c, n: {k: v / n for k, v in c.items()}  # noqa: E731
    r = per(rhs, interior)
    s = per(step, interior * stages)
    return {"rhs": r, "stage": s, "rhs_flops": _flops(r), "stage_flops": _flops(s),
            "box": [mx, my, mz], "stages": stages}
