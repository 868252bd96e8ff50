"""Generates the immersed-boundary fixtures in tests/golden/ibm/*.npz.

Each fixture holds a seeded periodic grid with a triangulated sphere
(workloads.sphere_surface), the conserved state, the surface velocities, and
what the REFERENCE's own code makes of them: ibm_search_advanced
(ibm_iso.c:87) sets nvert and builds the interpolation list,
ibm_interpolation_advanced (ibm_iso.c:2572) runs once on the state, and
RungeKutta with -imm 1 (solvers.c:223-294) advances full steps.  ibm_iso.c,
compgeom.c, variables.c and wallfunction.c are compiled unmodified against the
serial PETSc shim with the rest of the hot path (oracle/_ref).  Run from the
repo root in a checkout that has the reference sources:

    python tests/golden/make_ibm_golden.py [case ...]

The reference builds a list only with -isothermal 1 or 2 (ibm_iso.c:534-760);
the "iso0" case reuses the list of an isothermal-1 search for an
interpolation with -isothermal 0 (d rho / dn = 0).  Two cases have
non-periodic faces: after the interpolation FormBCS(user, 0) rewrites some
boundary nodes of Q without their pressure, and no EqOfState follows, so the
next step's first stage reads that carried pressure (solvers.c:279-288).

Arrays per fixture: coords, q, nvert, the surface (x, y, z, nv1..nv3,
nf_x..nf_z), u / uold (vertex velocities), info_i / info_r (the list, 13 ints
and 11 doubles per entry in the list's order), q_interp / p_interp (Q and P
after one interpolation with Add_dUndt = 1, at the listed nodes in list
order; every other node keeps its Q) and q_steps (Q after `steps` immersed
time steps from q).
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "ibm")
sys.path.insert(0, REPO)

import oracle as O  # noqa: E402
from chimera_comp_les_b200 import workloads as W  # noqa: E402

N = (16, 14, 15)
CASES = {
    # name: (config kwargs, list config override, seed, steps)
    "sphere_noslip": (dict(les=0, inviscid=0, fluxorder=3, ren=300., ma=0.3, pr=0.71, dt=0.002, isothermal=1),
                      None, 1, 2),
    "sphere_les_freeslip_wf3": (dict(les=1, inviscid=0, fluxorder=2, ren=500., ma=0.3, pr=0.71, dt=0.002,
                                     isothermal=1, wallfunction=3), None, 2, 2),
    "sphere_inviscid_twoD2": (dict(les=0, inviscid=1, fluxorder=3, ma=0.3, dt=0.002, isothermal=1, twoD=2),
                              None, 3, 2),
    "sphere_iso0": (dict(les=0, inviscid=0, fluxorder=3, ren=300., ma=0.3, pr=0.71, dt=0.002, isothermal=0),
                    dict(isothermal=1), 4, 2),
    # inflow / outflow along k (bctype 45), the sphere benchmark's k faces
    "sphere_kflow45": (dict(les=0, inviscid=0, fluxorder=3, ren=300., ma=0.3, pr=0.71, dt=0.002, isothermal=1,
                            bctype=(7, 7, 7, 7, 45, 45)), None, 5, 3),
    # slip walls in j, outflow 44 in k, LES
    "sphere_les_walls44": (dict(les=1, inviscid=0, fluxorder=3, ren=400., ma=0.3, pr=0.71, dt=0.002, isothermal=1,
                                bctype=(7, 7, 3, 3, 44, 44)), None, 6, 3),
    # the dynamic Smagorinsky model (-les 2) around the body
    "sphere_les2_dynamic": (dict(les=2, inviscid=0, fluxorder=3, ren=400., ma=0.3, pr=0.71, dt=0.002, isothermal=1,
                                 max_cs=0.1), None, 7, 3),
    # the shock sensor, which reads the pressure carried from the interpolation
    # at the first stage of every step after the first
    "sphere_les_sensor": (dict(les=1, inviscid=0, fluxorder=3, ren=400., ma=0.3, pr=0.71, dt=0.002, isothermal=1,
                               calc_sigma=1, s_x=0.7, s_y=0.8, s_z=0.9, s_y_min=0.05, sigma_thrsh=1e-3), None, 8, 3),
    # the characteristic isothermal wall (-isothermal 2, ibm_iso.c:2744-2786)
    # with a wall temperature of 1.2
    "sphere_iso2": (dict(les=0, inviscid=0, fluxorder=3, ren=300., ma=0.3, pr=0.71, dt=0.002, isothermal=2,
                         twall=1.2), None, 9, 3),
    # the k-lo inflow codes that read the node coordinates: the characteristic
    # cos^2 inlet 52 with slip j walls, the power-law inlet 47 (step index)
    "sphere_inflow52": (dict(les=1, inviscid=0, fluxorder=3, ren=400., ma=0.3, pr=0.71, dt=0.002, isothermal=1,
                             bctype=(7, 7, 3, 3, 52, 45)), None, 10, 3),
    "sphere_inflow47": (dict(les=0, inviscid=0, fluxorder=3, ren=400., ma=0.3, pr=0.71, dt=0.002, isothermal=1,
                             bctype=(7, 7, 7, 7, 47, 45)), None, 11, 3),
}


def make(name, spec):
    kw, list_kw, seed, steps = spec
    coords = W.periodic_grid(N, 2 * np.pi, amp=0.03)
    if kw.get("bctype", (7,) * 6)[4] in (52, 47):
        # y from about 1 to 10.4: 47's power law (y/8)^0.1428 needs y > 0, and
        # both of its branches (y < 8, y >= 8) are met
        coords[..., 1] = 1.5 * coords[..., 1] + 1.0
    shape = coords.shape[:3]
    cfg = O.Config(mx=N[0] + 2, my=N[1] + 2, mz=N[2] + 2, immersed=1, **kw)
    ctr = coords[shape[0] // 2, shape[1] // 2, shape[2] // 2]
    surf = W.sphere_surface(1.6, ctr, 3)
    n_v = len(surf["x"])
    rng = np.random.default_rng(seed)
    # a slowly accelerating surface: d(Un)/dt = O(0.1), pressures stay positive
    u = rng.normal(size=(n_v, 3)) * 0.02
    uold = u + rng.normal(size=(n_v, 3)) * 2e-4
    q = W.random_smooth_state(shape, seed=seed)

    scfg = O.Config(**{**cfg.__dict__, **(list_kw or {})})
    ref = O.RefOracle(scfg, coords)
    ref.ibm_setup(surf)
    nvert, info = ref.ibm_search()

    ref = O.RefOracle(cfg, coords)
    ref.ibm_setup(surf)
    ref.ibm_set_list(info)
    ref.ibm_set_velocity(u, uold)
    ref.set_nvert(nvert)
    ref.set_state(q)
    ref.ibm_interpolate(1)
    q_interp, p_interp = ref.Q(), ref.P()

    ref = O.RefOracle(cfg, coords)
    ref.ibm_setup(surf)
    ref.ibm_set_list(info)
    ref.ibm_set_velocity(u, uold)
    ref.set_nvert(nvert)
    ref.set_state(q)
    ref.steps(steps)
    q_steps = ref.Q()

    assert np.isfinite(q_interp).all() and np.isfinite(q_steps).all(), name
    # the interpolation writes Q and P at the listed nodes only
    k, j, i = info["nk"], info["nj"], info["ni"]
    rest = np.ones(shape, dtype=bool)
    rest[k, j, i] = False
    assert np.array_equal(q_interp[rest], q[rest])
    iv, rv = O.ibm_info_to_flat(info)
    meta = dict(name=name, config={a: (list(v) if isinstance(v, tuple) else v) for a, v in cfg.__dict__.items()},
                steps=steps, entries=int(info.size),
                generator="reference ibm_iso.c/compgeom.c/variables.c/wallfunction.c + hot path via oracle/_ref")
    os.makedirs(OUT, exist_ok=True)
    np.savez_compressed(os.path.join(OUT, f"{name}.npz"), coords=coords, q=q, nvert=nvert, u=u, uold=uold,
                        info_i=iv, info_r=rv, q_interp=q_interp[k, j, i], p_interp=p_interp[k, j, i], q_steps=q_steps,
                        meta=np.array(json.dumps(meta)), **{a: np.asarray(v) for a, v in surf.items()})
    print("wrote", name, "entries", info.size)


if __name__ == "__main__":
    # python tests/golden/make_ibm_golden.py [name ...]: the named cases, else all
    for n in sys.argv[1:] or list(CASES):
        make(n, CASES[n])
