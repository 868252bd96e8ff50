"""Shared helpers for the tests: golden fixtures and oracle/GPU runners."""
import glob
import json
import os

import numpy as np

import oracle as O

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# Parity bar for the FP64 form against the oracle: per conserved field,
# relative L2 <= 1e-12.
RTOL_L2 = 1e-12


def golden_names():
    return sorted(os.path.splitext(os.path.basename(p))[0] for p in glob.glob(os.path.join(GOLDEN_DIR, "*.npz")))


def load_golden(name):
    d = np.load(os.path.join(GOLDEN_DIR, name + ".npz"))
    meta = json.loads(str(d["meta"]))
    cfgd = dict(meta["config"])
    cfgd["bctype"] = tuple(cfgd["bctype"])
    cfg = O.Config(**cfgd)
    return cfg, meta, {k: d[k] for k in d.files if k != "meta"}


def oracle_run(cfg, coords, q, nvert, steps=0):
    """Restatement: metrics, (nut), rhs at istage 0, Q after `steps` steps."""
    ora = O.Oracle(cfg)
    met = ora.metrics(O.to_padded(cfg, coords))
    nvp = ora.fill_ghosts(O.to_padded(cfg, nvert))
    st = ora.initial_state(q)
    sig = ora.sigma(st["q"]) if cfg.les else None
    nut = ora.zeros(1)
    out = {"metrics": {k: O.from_padded(v) for k, v in met.items()}}
    if cfg.les and not cfg.inviscid:
        ora.eddy_viscosity(st["q"], met, nvp, nut)
        out["nut"] = O.from_padded(nut)[..., 0]
    out["rhs"] = O.from_padded(ora.rhs(st["q"], met, nvp, nut, sig))
    if steps:
        st = ora.initial_state(q)
        ora.steps(steps, st, met, nvp)
        out["q_steps"] = O.from_padded(st["q"])
    return out


def gpu_block(cfg, precision="fp64"):
    from chimera_comp_les_b200 import Block
    return Block(cfg.mx, cfg.my, cfg.mz, bctype=tuple(cfg.bctype), les=cfg.les, inviscid=cfg.inviscid,
                 fluxorder=cfg.fluxorder, eno_order=cfg.eno_order, central=cfg.central,
                 isothermal=cfg.isothermal, s_x=cfg.s_x, s_y=cfg.s_y, s_z=cfg.s_z, ren=cfg.ren, ma=cfg.ma,
                 pr=cfg.pr, gamma=cfg.gamma, dt=cfg.dt, st=cfg.st, cs_const=cfg.cs_const, ci=cfg.ci,
                 ratio=cfg.ratio, precision=precision, calc_sigma=cfg.calc_sigma, s_x_min=cfg.s_x_min,
                 s_y_min=cfg.s_y_min, s_z_min=cfg.s_z_min, sigma_thrsh=cfg.sigma_thrsh, flux=cfg.flux)


def per_field_rel_l2(a, b):
    return [O.rel_l2(a[..., f], b[..., f]) for f in range(a.shape[-1])]
