"""Generates the golden fixtures in tests/golden/*.npz.

Each fixture holds seeded inputs (coordinates, conserved state, nvert mask)
and the outputs of the REFERENCE's own code for them: rhs.c / les.c /
metrics.c / solvers.c compiled unmodified against the serial PETSc shim
(oracle/_ref).  Run from the repo root in a checkout that has the reference
sources (they are read only by this script, never by the tests):

    python tests/golden/make_golden.py

Outputs per fixture:
  metrics_csi/eta/zet/aj : FormMetrics result (global, natural order)
  nut                    : Compute_eddy_viscosity_LES after CalcUCat (LES cases)
  rhs                    : formRHS(istage=0) on the uploaded state
  q_steps                : Q after `steps` full time steps from the uploaded state
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

import oracle as O  # noqa: E402
from chimera_comp_les_b200 import workloads as W  # noqa: E402

CASES = {
    # name: (N(x,y,z), amp, seed, config kwargs, mask, steps)
    "inviscid_weno3": ((10, 11, 9), 0.05, 1, dict(les=0, inviscid=1, fluxorder=3, dt=0.004), False, 3),
    "viscous_muscl": ((10, 9, 11), 0.05, 2, dict(les=0, inviscid=0, fluxorder=2, ren=200., ma=0.3, pr=0.71, dt=0.004), True, 3),
    "les_muscl_sigma1": ((11, 10, 9), 0.05, 3, dict(les=1, inviscid=0, fluxorder=2, ren=1600., ma=0.3, pr=0.71, dt=0.004), False, 3),
    "les_weno_blend": ((9, 10, 11), 0.05, 4, dict(les=1, inviscid=0, fluxorder=3, s_x=0.3, s_y=0.6, s_z=0.8, ren=400., ma=0.3, pr=0.71, dt=0.004), True, 2),
    "les_first_order_central3": ((10, 10, 10), 0.03, 5, dict(les=1, inviscid=0, fluxorder=1, central=3, eno_order=3, ren=300., ma=0.3, pr=0.71, dt=0.003), True, 2),
    # dynamic Smagorinsky (Compute_Smagorinsky_Constant_1 with -les 2)
    "les2_dynamic_weno_mask": ((11, 9, 10), 0.05, 6, dict(les=2, inviscid=0, fluxorder=3, ren=800., ma=0.3, pr=0.71, dt=0.003, max_cs=0.1), True, 3),
}


def nvert_blob(shape, seed):
    rng = np.random.default_rng(seed)
    mz, my, mx = shape
    z, y, x = np.meshgrid(np.arange(mz), np.arange(my), np.arange(mx), indexing="ij")
    c = rng.uniform(4, min(shape) - 4, 3)
    r = np.sqrt((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2)
    nv = np.zeros(shape)
    nv[r < 2.5] = 1.0   # interface band (ibm_iso.c:765: 1 + ibi/1000)
    nv[r < 1.6] = 3.0   # solid (3 + ibi/1000)
    return nv


def make(name, spec):
    (nx, ny, nz), amp, seed, kw, mask, steps = spec
    coords = W.periodic_grid((nx, ny, nz), 2 * np.pi, amp=amp)
    shape = coords.shape[:3]
    cfg = O.Config(mx=nx + 2, my=ny + 2, mz=nz + 2, **kw)
    q = W.random_smooth_state(shape, seed=seed)
    nv = nvert_blob(shape, seed + 100) if mask else np.zeros(shape)

    ref = O.RefOracle(cfg, coords)
    ref.set_nvert(nv)
    ref.set_state(q)
    met = ref.metrics_local()
    out = {}
    for k in ("csi", "eta", "zet", "aj"):
        out["metrics_" + k] = O.from_padded(O.local_to_padded(cfg, met[k], met[k].shape[-1]))
    if cfg.les and not cfg.inviscid:
        ref.calc_ucat()
        ref.eddy_viscosity()
        out["nut"] = ref.nut()
    out["rhs"] = ref.rhs(0)
    ref2 = O.RefOracle(cfg, coords)
    ref2.set_nvert(nv)
    ref2.set_state(q)
    ref2.steps(steps)
    out["q_steps"] = ref2.Q()
    meta = dict(name=name, config={k: (list(v) if isinstance(v, tuple) else v) for k, v in cfg.__dict__.items()},
                steps=steps, generator="reference rhs.c/les.c/metrics.c/solvers.c via oracle/_ref (PETSc shim)")
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), coords=coords, q=q, nvert=nv,
                        meta=np.array(json.dumps(meta)), **out)
    print("wrote", name)


if __name__ == "__main__":
    for n, s in CASES.items():
        make(n, s)
