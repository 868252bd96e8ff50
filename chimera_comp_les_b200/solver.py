"""Host-side mirror of the reference's hot-path interface over the C-ABI.

``Block`` is one DMDA block of the reference resident on a B200.  Its methods
carry the names of the reference functions they replace and take/return the
arrays behind the reference's PETSc global Vecs as numpy arrays in natural
AoS order (mz, my, mx, ncomp):

  FormMetrics(coor)                  metrics.c:3      (cb_set_grid)
  SetInitialCondition(Q)             rhs.c:420-433    (cb_upload_state)
  formRHS(istage)                    rhs.c:4703       (cb_rhs)
  CalcUCat()                         rhs.c:1322       (cb_calc_ucat)
  Compute_eddy_viscosity_LES()       les.c:1477       (cb_eddy_viscosity)
  RungeKutta(nsteps) / Flow_Solver   solvers.c:13,223 (cb_rk_step)
  EqOfState()                        rhs.c:4820       (pressure download)
  ibm_interpolation_advanced(ibi)    ibm_iso.c:2572   (cb_ibm_interpolate)

Immersed bodies: ``set_ibm_surface`` / ``set_ibm_velocity`` / ``set_ibm_list``
hand over what the reference's host search built (IBMNodes and
user->ibmlist[ibi]); every ``RungeKutta`` step then interpolates each body
after the stages and applies FormBCS(user, 0) on the device
(solvers.c:282-288).

Options may be given as the reference's command-line flags via
``Block.from_options``.
"""
from __future__ import annotations

import ctypes as C
import shlex
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import CbConfig, ChimeraError, dptr

_OPT_MAP = {
    "-les": ("les", int), "-inv": ("inviscid", int), "-fluxorder": ("fluxorder", int),
    "-ENOorder": ("eno_order", int), "-central": ("central", int), "-isothermal": ("isothermal", int),
    "-s_x": ("s_x", float), "-s_y": ("s_y", float), "-s_z": ("s_z", float), "-ren": ("ren", float),
    "-Ma": ("ma", float), "-Pr": ("pr", float), "-gamma": ("gamma", float), "-dt": ("dt", float),
    "-calc_sigma": ("calc_sigma", int), "-s_x_min": ("s_x_min", float), "-s_y_min": ("s_y_min", float),
    "-s_z_min": ("s_z_min", float), "-sigma_thrsh": ("sigma_thrsh", float), "-max_cs": ("max_cs", float),
    "-Twall": ("twall", float), "-twoD": ("twod", int), "-i_homo_filter": ("i_homo_filter", int),
    "-j_homo_filter": ("j_homo_filter", int), "-k_homo_filter": ("k_homo_filter", int),
    "-testfilter_ik": ("testfilter_ik", int), "-visT": ("visT", int), "-Tref": ("tref", float),
    "-ABC": ("abc", int),
}


def _f64(a: np.ndarray, shape) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float64)
    if a.shape != tuple(shape):
        a = a.reshape(shape)
    return a


class Block:
    """One curvilinear block of the reference's solver, resident on one GPU."""

    def __init__(self, mx: int, my: int, mz: int, bctype: Sequence[int] = (7, 7, 7, 7, 7, 7), les: int = 0,
                 inviscid: int = 0, fluxorder: int = 3, eno_order: int = 2, central: int = 2,
                 isothermal: int = 0, s_x: float = 1.0, s_y: float = 1.0, s_z: float = 1.0,
                 ren: float = 3000.0, ma: float = 2.81, pr: float = 0.72, gamma: float = 1.4,
                 dt: float = 0.01, st: float = 1.0, cs_const: float = 0.03, ci: float = 0.06,
                 ratio: float = 0.0, precision: str = "fp64", device: int = 0, calc_sigma: int = 0,
                 s_x_min: float = 0.0, s_y_min: float = 0.0, s_z_min: float = 0.0, sigma_thrsh: float = 1e-5,
                 flux: str = "rusanov", max_cs: float = 0.05, twall: float = 1.0, twod: int = 0,
                 i_homo_filter: int = 0, j_homo_filter: int = 0, k_homo_filter: int = 0, testfilter_ik: int = 0,
                 visT: int = 0, tref: float = 273.15, abc: int = 0, weno_order: int = 3):
        self.lib = _lib.load()
        cfg = CbConfig()
        self.lib.cb_config_default(C.byref(cfg), mx, my, mz)
        cfg.bctype = (C.c_int * 6)(*bctype)
        for k, v in dict(les=les, inviscid=inviscid, fluxorder=fluxorder, eno_order=eno_order, central=central,
                         isothermal=isothermal, s_x=s_x, s_y=s_y, s_z=s_z, ren=ren, ma=ma, pr=pr, gamma=gamma,
                         dt=dt, st=st, cs_const=cs_const, ci=ci, ratio=ratio, device=device, calc_sigma=calc_sigma,
                         s_x_min=s_x_min, s_y_min=s_y_min, s_z_min=s_z_min, sigma_thrsh=sigma_thrsh,
                         max_cs=max_cs, twall=twall, twod=twod, i_homo_filter=i_homo_filter,
                         j_homo_filter=j_homo_filter, k_homo_filter=k_homo_filter,
                         testfilter_ik=testfilter_ik, visT=visT, tref=tref, abc=abc,
                         weno_order=weno_order).items():
            setattr(cfg, k, v)
        cfg.flux = {"rusanov": 0, "roe": 1}[flux] if isinstance(flux, str) else int(flux)
        cfg.precision = {"fp64": _lib.CB_FP64, "mixed": _lib.CB_MIXED}[precision]
        self.cfg = cfg
        self.shape = (mz, my, mx)
        self._ctx = C.c_void_p()
        rc = self.lib.cb_create(C.byref(cfg), C.byref(self._ctx))
        if rc != 0:
            raise ChimeraError(rc, "cb_create failed (see stderr)")

    @classmethod
    def from_options(cls, mx: int, my: int, mz: int, options: str, bctype=(7, 7, 7, 7, 7, 7), **kw) -> "Block":
        """Build from the reference's option flags, e.g. "-les 1 -fluxorder 2 -ren 1600"."""
        toks = shlex.split(options)
        args = dict(kw)
        for name, val in zip(toks[::2], toks[1::2]):
            if name in _OPT_MAP:
                key, typ = _OPT_MAP[name]
                args[key] = typ(val)
        return cls(mx, my, mz, bctype=bctype, **args)

    # ------------------------------------------------------------ helpers --
    def _check(self, rc: int):
        if rc != 0:
            msg = self.lib.cb_last_error(self._ctx)
            raise ChimeraError(rc, msg.decode() if msg else "")

    @property
    def nnodes(self) -> int:
        mz, my, mx = self.shape
        return mx * my * mz

    @property
    def interior_nodes(self) -> int:
        return int(self.lib.cb_interior_nodes(self._ctx))

    @property
    def stages(self) -> int:
        return int(self.lib.cb_stages(self._ctx))

    @property
    def launches_per_step(self) -> int:
        return int(self.lib.cb_launches_per_step(self._ctx))

    @property
    def stream(self) -> int:
        return int(self.lib.cb_stream(self._ctx) or 0)

    # ----------------------------------------------------- reference calls --
    def FormMetrics(self, coor: np.ndarray):
        c = _f64(coor, self.shape + (3,))
        self._check(self.lib.cb_set_grid(self._ctx, dptr(c)))

    def set_metrics(self, csi, eta, zet, aj):
        a = [_f64(x, self.shape + (3,)) for x in (csi, eta, zet)] + [_f64(aj, self.shape)]
        self._check(self.lib.cb_set_metrics(self._ctx, *[dptr(x) for x in a]))

    def metrics(self):
        """(csi, eta, zet, aj) as resident on the device, natural AoS order."""
        csi, eta, zet = (np.empty(self.shape + (3,)) for _ in range(3))
        aj = np.empty(self.shape)
        self._check(self.lib.cb_get_metrics(self._ctx, dptr(csi), dptr(eta), dptr(zet), dptr(aj)))
        return csi, eta, zet, aj

    def set_nvert(self, nvert: np.ndarray):
        n = _f64(nvert, self.shape)
        self._check(self.lib.cb_set_nvert(self._ctx, dptr(n)))

    def SetInitialCondition(self, q: np.ndarray):
        a = _f64(q, self.shape + (5,))
        self._check(self.lib.cb_upload_state(self._ctx, dptr(a)))
        self._check(self.lib.cb_sync(self._ctx))

    upload_state = SetInitialCondition

    # ------------------------------------------------------ immersed bodies --
    def set_ibm_surface(self, ibi: int, surface: dict):
        """IBMNodes of body ibi: nv1, nv2, nv3 (vertex indices per triangle),
        nf_x, nf_y, nf_z (unit normals) and x (for the vertex count)."""
        tri = [np.ascontiguousarray(surface[k], dtype=np.int32) for k in ("nv1", "nv2", "nv3")]
        nf = [np.ascontiguousarray(surface[k], dtype=np.float64) for k in ("nf_x", "nf_y", "nf_z")]
        n_v = int(surface["n_v"]) if "n_v" in surface else len(surface["x"])
        self._check(self.lib.cb_ibm_set_surface(self._ctx, ibi, n_v, len(tri[0]), *[t.ctypes.data for t in tri],
                                                *[dptr(a) for a in nf]))

    def set_ibm_velocity(self, ibi: int, u: np.ndarray, uold: np.ndarray):
        """Vertex velocities ibm->u and ibm->uold, shape (n_v, 3)."""
        u = np.ascontiguousarray(u, dtype=np.float64)
        uold = np.ascontiguousarray(uold, dtype=np.float64)
        self._check(self.lib.cb_ibm_set_velocity(self._ctx, ibi, dptr(u), dptr(uold)))

    def set_ibm_list(self, ibi: int, info: np.ndarray, coor: np.ndarray):
        """Interpolation list of body ibi (structured array of _lib.IBM_INFO_DTYPE,
        in the reference's list order) and the node coordinates."""
        a = np.ascontiguousarray(info, dtype=_lib.IBM_INFO_DTYPE)
        c = _f64(coor, self.shape + (3,))
        self._check(self.lib.cb_ibm_set_list(self._ctx, ibi, a.size, a.ctypes.data if a.size else None, dptr(c)))

    def ibm_count(self, ibi: int) -> int:
        return int(self.lib.cb_ibm_count(self._ctx, ibi))

    def set_ibm_options(self, twoD: int = 0, wallfunction: int = 0):
        self._check(self.lib.cb_ibm_set_options(self._ctx, twoD, wallfunction))

    def ibm_ustar(self, ibi: int = 0) -> np.ndarray:
        """u_tau of every entry of body ibi's list from the last sweep with
        -wallfunction 2 (cb_ibm_get_ustar)."""
        out = np.zeros(max(self.lib.cb_ibm_count(self._ctx, ibi), 0))
        self._check(self.lib.cb_ibm_get_ustar(self._ctx, ibi, out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def ibm_interpolation_advanced(self, ibi: int = 0, Add_dUndt: int = 1):
        self._check(self.lib.cb_ibm_interpolate(self._ctx, ibi, Add_dUndt))

    def formRHS(self, istage: int = 0) -> np.ndarray:
        out = np.empty(self.shape + (5,))
        self._check(self.lib.cb_rhs(self._ctx, istage, dptr(out)))
        return out

    def cfl_dt(self, cfl: float):
        """(dt, lambda_max) for the CFL number `cfl` on the current state."""
        dt, lam = C.c_double(), C.c_double()
        self._check(self.lib.cb_cfl_dt(self._ctx, float(cfl), C.byref(dt), C.byref(lam)))
        return dt.value, lam.value

    def autotune(self, candidates=None):
        """Time the stage kernel per k-chunk candidate and keep the fastest
        (k-chunk 0: balanced segments, one range of tile-column planes per
        resident CTA).  Returns (best k-chunk, {k-chunk: ms})."""
        cand = list(candidates or [])
        ca = (C.c_int * max(len(cand), 1))(*cand)
        cap = max(len(cand), self.shape[0] + 1)
        ms = (C.c_double * cap)()
        nout, best = C.c_int(cap), C.c_int()
        self._check(self.lib.cb_autotune(self._ctx, len(cand), ca, ms, C.byref(nout), C.byref(best)))
        if cand:
            keys = cand
        else:
            nk, keys, last = self.shape[0] - 2, [], -1
            for kc in range(nk, 3, -1):
                ch = -(-nk // kc)
                if ch != last:
                    keys.append(kc)
                    last = ch
            keys.append(0)  # balanced segments
        return best.value, {k: ms[i] for i, k in enumerate(keys[:nout.value])}

    def CalcUCat(self):
        self._check(self.lib.cb_calc_ucat(self._ctx))

    def Compute_eddy_viscosity_LES(self):
        self._check(self.lib.cb_eddy_viscosity(self._ctx))

    def CS(self) -> np.ndarray:
        """The dynamic Smagorinsky coefficient user->CS (-les 2)."""
        out = np.empty(self.shape)
        self._check(self.lib.cb_get_cs(self._ctx, dptr(out)))
        return out

    def nu_t(self) -> np.ndarray:
        out = np.empty(self.shape)
        self._check(self.lib.cb_get_nut(self._ctx, dptr(out)))
        return out

    def upload_async(self, q: np.ndarray) -> None:
        """cb_upload_state_async: Q (natural AoS, ideally pinned host memory)
        as the new state; returns after enqueueing.  Keep q unchanged until
        join_transfers() and sync()."""
        assert q.dtype == np.float64 and q.flags.c_contiguous and q.size == 5 * self.nnodes
        self._check(self.lib.cb_upload_state_async(self._ctx, q.ctypes.data))

    def download_async(self, q_out: np.ndarray) -> None:
        """cb_download_state_async: Q into q_out after the work enqueued so far;
        returns after enqueueing (q_out is valid after join_transfers() and sync())."""
        assert q_out.dtype == np.float64 and q_out.flags.c_contiguous and q_out.size == 5 * self.nnodes
        self._check(self.lib.cb_download_state_async(self._ctx, q_out.ctypes.data))

    def join_transfers(self) -> None:
        """cb_join_transfers: later work on the context's stream follows every copy."""
        self._check(self.lib.cb_join_transfers(self._ctx))

    def set_time_index(self, ti: int) -> None:
        """user->ti of the last completed step (the next RungeKutta step is
        ti + 1); read by the k-lo inflow code 47 (cb_set_time_index)."""
        self._check(self.lib.cb_set_time_index(self._ctx, int(ti)))

    def RungeKutta(self, nsteps: int = 1, sync: bool = True):
        self._check(self.lib.cb_rk_step(self._ctx, int(nsteps)))
        if sync:
            self.sync()

    Flow_Solver = RungeKutta

    def sync(self):
        self._check(self.lib.cb_sync(self._ctx))

    def Q(self) -> np.ndarray:
        out = np.empty(self.shape + (5,))
        self._check(self.lib.cb_download_state(self._ctx, dptr(out), None))
        return out

    def EqOfState(self) -> np.ndarray:
        q = np.empty(self.shape + (5,))
        p = np.empty(self.shape)
        self._check(self.lib.cb_download_state(self._ctx, dptr(q), dptr(p)))
        return p

    def download(self, q_out: np.ndarray, p_out: Optional[np.ndarray] = None):
        self._check(self.lib.cb_download_state(self._ctx, dptr(q_out), dptr(p_out)))

    # --------------------------------------------------------------- timing --
    def timing(self, on: bool):
        self._check(self.lib.cb_timing_enable(self._ctx, 1 if on else 0))

    def timing_read(self):
        a, b = C.c_double(), C.c_double()
        na, nb = C.c_int(), C.c_int()
        self._check(self.lib.cb_timing_read(self._ctx, C.byref(a), C.byref(na), C.byref(b), C.byref(nb)))
        return a.value, na.value, b.value, nb.value

    def close(self):
        if self._ctx:
            self.lib.cb_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
