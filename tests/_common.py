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
    if cfg.bctype[4] in (52, 47):  # the inflow codes read the node coordinates
        ora.set_coordinates(O.to_padded(cfg, coords))
    met = ora.metrics(O.to_padded(cfg, coords))
    nvp = ora.fill_ghosts(O.to_padded(cfg, nvert))
    st = ora.initial_state(q)
    sig = ora.sigma(st["q"]) if cfg.les else None
    nut = ora.zeros(1)
    out = {"metrics": {k: O.from_padded(v) for k, v in met.items()}}
    if cfg.les >= 2 and cfg.les != 10 and not cfg.inviscid:  # CalcUCat on the same state, then the dynamic model
        cs = ora.dynamic_smagorinsky(st["q"], st["q"], met, nvp)
        ora.eddy_viscosity_dyn(st["q"], st["q"], met, nvp, cs, nut)
        out["nut"] = O.from_padded(nut)[..., 0]
        out["cs"] = O.from_padded(cs)[..., 0]
    elif cfg.les and cfg.les != 10 and not cfg.inviscid:
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
                 s_y_min=cfg.s_y_min, s_z_min=cfg.s_z_min, sigma_thrsh=cfg.sigma_thrsh, flux=cfg.flux,
                 max_cs=cfg.max_cs, twall=cfg.twall, twod=cfg.twoD, i_homo_filter=cfg.i_homo_filter,
                 j_homo_filter=cfg.j_homo_filter, k_homo_filter=cfg.k_homo_filter, testfilter_ik=cfg.testfilter_ik,
                 visT=cfg.visT, tref=cfg.tref, abc=cfg.abc, weno_order=cfg.weno_order)


def per_field_rel_l2(a, b):
    return [O.rel_l2(a[..., f], b[..., f]) for f in range(a.shape[-1])]


# ------------------------------------------------------------ immersed body --
IBM_DIR = os.path.join(GOLDEN_DIR, "ibm")
SURFACE_KEYS = ("x", "y", "z", "nv1", "nv2", "nv3", "nf_x", "nf_y", "nf_z")


def ibm_golden_names():
    return sorted(os.path.splitext(os.path.basename(p))[0] for p in glob.glob(os.path.join(IBM_DIR, "*.npz")))


def load_ibm_golden(name):
    """cfg, meta, arrays, list (O.IBM_INFO_DTYPE), surface dict of one fixture."""
    d = np.load(os.path.join(IBM_DIR, name + ".npz"))
    meta = json.loads(str(d["meta"]))
    cfgd = dict(meta["config"])
    cfgd["bctype"] = tuple(cfgd["bctype"])
    cfg = O.Config(**cfgd)
    g = {k: d[k] for k in d.files if k != "meta"}
    info = O.ibm_info_from_flat(g["info_i"], g["info_r"])
    surf = {k: g[k] for k in SURFACE_KEYS}
    return cfg, meta, g, info, surf


def synthetic_ibm_list(cfg, coords, n_elmt, seed, radius=3.0, dup=12, on_surface=4):
    """An interpolation list over a spherical band of nodes around the block's
    centre: donors within two nodes (often other listed nodes, so sweeps chain),
    random positive weights summing to one, ~10% entries without a surface
    element, `on_surface` entries whose node is its own interception point (the
    element-normal fallback), and `dup` nodes listed a second time later on
    (the later entry wins)."""
    rng = np.random.default_rng(seed)
    mz, my, mx = coords.shape[:3]
    z, y, x = np.meshgrid(np.arange(mz), np.arange(my), np.arange(mx), indexing="ij")
    c = np.array([mx, my, mz]) / 2.0
    r = np.sqrt((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2)
    band = np.argwhere((r > radius - 0.8) & (r < radius + 0.8))
    n = len(band)
    info = np.zeros(n + dup, dtype=O.IBM_INFO_DTYPE)
    rows = np.concatenate([np.arange(n), rng.choice(n, dup, replace=False)])
    for e, b in enumerate(rows):
        k, j, i = band[b]
        info[e]["ni"], info[e]["nj"], info[e]["nk"] = i, j, k
        for t, (a, bb, cc) in enumerate((("i1", "j1", "k1"), ("i2", "j2", "k2"), ("i3", "j3", "k3"))):
            off = rng.integers(-2, 3, size=3)
            if not off.any():
                off[0] = 1
            info[e][a], info[e][bb], info[e][cc] = i + off[0], j + off[1], k + off[2]
        w = rng.uniform(0.1, 1.0, 3)
        w /= w.sum()
        info[e]["cr1"], info[e]["cr2"], info[e]["cr3"] = w
        s = rng.uniform(0.1, 1.0, 3)
        s /= s.sum()
        info[e]["cs1"], info[e]["cs2"], info[e]["cs3"] = s
        info[e]["cell"] = -1 if rng.random() < 0.1 else rng.integers(0, n_elmt)
        info[e]["d_s"] = rng.uniform(0.05, 0.3)
        info[e]["d_i"] = rng.uniform(0.1, 0.5)
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        info[e]["pmin"] = coords[k, j, i] - d * info[e]["d_s"]
    for e in rng.choice(n, on_surface, replace=False):
        k, j, i = info[e]["nk"], info[e]["nj"], info[e]["ni"]
        info[e]["pmin"] = coords[k, j, i]
    return info


def gpu_ibm_block(cfg, coords, nvert, q, surf, info, u=None, uold=None, precision="fp64"):
    b = gpu_block(cfg, precision)
    b.FormMetrics(coords)
    b.set_nvert(nvert)
    b.SetInitialCondition(q)
    b.set_ibm_options(twoD=cfg.twoD, wallfunction=cfg.wallfunction)
    b.set_ibm_surface(0, surf)
    if u is not None:
        b.set_ibm_velocity(0, u, uold)
    b.set_ibm_list(0, info, coords)
    return b
