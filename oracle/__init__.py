"""CPU oracle for the compressible RHS + SSP-RK stage update.

TEST INFRASTRUCTURE ONLY.  Only tests/, the smoke entry point and the
CPU-baseline leg of bench.py import this package, and only as the checker.

Two CPU implementations live here:

* ``Oracle`` -- the C restatement in ``oracle/src/cb_oracle.c`` (built into
  ``oracle/_build/liboracle.so`` from committed sources; gcc builds it on
  demand).
* ``RefOracle`` -- the reference's own ``rhs.c``, ``les.c``, ``metrics.c`` and
  ``solvers.c`` compiled unmodified against the serial PETSc shim into
  ``oracle/_ref/libchimera_ref.so`` (needs the reference checkout to build; a
  prebuilt copy travels with the working tree).

Array conventions (numpy):
  natural AoS : shape (mz, my, mx, ncomp) -- the reference's PETSc global Vec
  padded SoA  : shape (ncomp, mz+4, my+4, mx+4) -- node (i,j,k) at [.., k+2, j+2, i+2]
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(_HERE, "_build", "liboracle.so")
ORACLE_COUNT_SO = os.path.join(_HERE, "_build", "liboracle_count.so")
REF_SO = os.path.join(_HERE, "_ref", "libchimera_ref.so")
REF_SO_O3 = os.path.join(_HERE, "_ref", "libchimera_ref_O3.so")
# the same objects plus the reference's main.c: its checkpoint writer/reader
REF_IO_SO = os.path.join(_HERE, "_ref", "libchimera_ref_io.so")
# the reference checkout: CHIMERA_REF_DIR, else a sibling directory of this
# repository named "reference"
REF_SRC_DIR = os.environ.get("CHIMERA_REF_DIR") or os.path.normpath(os.path.join(_HERE, "..", "..", "reference"))


@dataclass
class Config:
    """Mirror of the reference options the hot path reads (main.c:716-801,
    init.c:45-103, rhs.c:2581-2585, 3242-3325)."""

    mx: int
    my: int
    mz: int
    bctype: Sequence[int] = (7, 7, 7, 7, 7, 7)
    les: int = 0
    inviscid: int = 0
    fluxorder: int = 3
    eno_order: int = 2
    central: int = 2
    isothermal: int = 0
    s_x: float = 1.0
    s_y: float = 1.0
    s_z: float = 1.0
    ren: float = 3000.0
    ma: float = 2.81
    pr: float = 0.72
    gamma: float = 1.4
    dt: float = 0.01
    st: float = 1.0
    cs_const: float = 0.03
    ci: float = 0.06
    ratio: float = 0.0
    calc_sigma: int = 0
    s_x_min: float = 0.0
    s_y_min: float = 0.0
    s_z_min: float = 0.0
    sigma_thrsh: float = 1e-5
    flux: int = 0  # 0 Rusanov (the reference's), 1 Roe (no reference counterpart)
    max_cs: float = 0.05  # -max_cs: clip of the dynamic Smagorinsky coefficient (les.c:151)
    twall: float = 1.0    # -Twall: characteristic isothermal wall temperature (rhs.c:486, 511)
    immersed: int = 0      # -imm: run the IB interpolation after the stages (solvers.c:282-288)
    wallfunction: int = 0  # -wallfunction: 0 noslip, 3 freeslip at IB nodes
    twoD: int = 0          # -twoD: 1/2/3 drops x/y/z from the IB normal and velocity
    i_homo_filter: int = 0  # -i/-j/-k_homo_filter: homogeneous averaging of the dynamic model (les.c:916-1115)
    j_homo_filter: int = 0
    k_homo_filter: int = 0
    testfilter_ik: int = 0  # -testfilter_ik: test-filter width 5^(1/3) filter widths (les.c:598)
    visT: int = 0           # -visT: Sutherland's law for the viscosity (rhs.c:1412-1414)
    tref: float = 273.15    # -Tref: its reference temperature (rhs.c:1410)
    abc: int = 0            # -ABC: absorbing layer of the shock sensor above plane k (rhs.c:3311)
    weno_order: int = 3     # 5: WENO5-JS (Jiang & Shu 1996) where its stencil fits; no reference counterpart
    ti0: int = 1            # user->ti of the first step (the k-lo inflow code 47 reads it)

    def ref_options(self) -> str:
        o = [
            ("-les", self.les), ("-inv", self.inviscid), ("-fluxorder", self.fluxorder),
            ("-ENOorder", self.eno_order), ("-central", self.central),
            ("-isothermal", self.isothermal), ("-s_x", repr(float(self.s_x))),
            ("-s_y", repr(float(self.s_y))), ("-s_z", repr(float(self.s_z))),
            ("-ren", repr(float(self.ren))), ("-Ma", repr(float(self.ma))),
            ("-Pr", repr(float(self.pr))), ("-gamma", repr(float(self.gamma))),
            ("-dt", repr(float(self.dt))), ("-visT", self.visT), ("-Tref", repr(float(self.tref))),
            ("-ABC", self.abc),
            ("-twoD", self.twoD), ("-TwoD", 0),
            ("-imm", self.immersed), ("-wallfunction", self.wallfunction), ("-max_cs", repr(float(self.max_cs))),
            ("-Twall", repr(float(self.twall))),
            ("-calc_sigma", self.calc_sigma), ("-s_x_min", repr(float(self.s_x_min))),
            ("-s_y_min", repr(float(self.s_y_min))), ("-s_z_min", repr(float(self.s_z_min))),
            ("-sigma_thrsh", repr(float(self.sigma_thrsh))),
            ("-i_homo_filter", self.i_homo_filter), ("-j_homo_filter", self.j_homo_filter),
            ("-k_homo_filter", self.k_homo_filter), ("-testfilter_ik", self.testfilter_ik),
        ]
        return " ".join(f"{k} {v}" for k, v in o)

    @property
    def padded_shape(self):
        return (self.mz + 4, self.my + 4, self.mx + 4)

    @property
    def nstages(self) -> int:
        return int(self.fluxorder)


class _CCfg(C.Structure):
    _fields_ = [
        ("mx", C.c_int), ("my", C.c_int), ("mz", C.c_int), ("bctype", C.c_int * 6),
        ("les", C.c_int), ("inviscid", C.c_int), ("fluxorder", C.c_int), ("eno_order", C.c_int),
        ("central", C.c_int), ("isothermal", C.c_int),
        ("s_x", C.c_double), ("s_y", C.c_double), ("s_z", C.c_double),
        ("ren", C.c_double), ("ma", C.c_double), ("pr", C.c_double), ("gamma", C.c_double),
        ("dt", C.c_double), ("st", C.c_double), ("cs_const", C.c_double), ("ci", C.c_double),
        ("ratio", C.c_double), ("calc_sigma", C.c_int),
        ("s_x_min", C.c_double), ("s_y_min", C.c_double), ("s_z_min", C.c_double), ("sigma_thrsh", C.c_double),
        ("flux", C.c_int), ("max_cs", C.c_double), ("twall", C.c_double), ("twod", C.c_int),
        ("i_homo_filter", C.c_int), ("j_homo_filter", C.c_int), ("k_homo_filter", C.c_int),
        ("testfilter_ik", C.c_int), ("visT", C.c_int), ("tref", C.c_double), ("abc", C.c_int),
        ("weno_order", C.c_int), ("coor_x", C.c_void_p), ("coor_y", C.c_void_p), ("ti0", C.c_int),
    ]


def _ccfg(cfg: Config) -> _CCfg:
    c = _CCfg()
    for f, _ in _CCfg._fields_:
        if f in ("coor_x", "coor_y"):
            continue  # set by Oracle.set_coordinates
        if f == "bctype":
            c.bctype = (C.c_int * 6)(*cfg.bctype)
        elif f == "twod":
            c.twod = cfg.twoD
        else:
            setattr(c, f, getattr(cfg, f))
    return c


# ---------------------------------------------------------------- layout --
def to_padded(cfg: Config, nat: np.ndarray) -> np.ndarray:
    """natural AoS (mz,my,mx,nc) -> padded SoA (nc,mz+4,my+4,mx+4); ghosts 0."""
    nat = np.asarray(nat, dtype=np.float64)
    if nat.ndim == 3:
        nat = nat[..., None]
    nc = nat.shape[-1]
    out = np.zeros((nc,) + cfg.padded_shape)
    out[:, 2:-2, 2:-2, 2:-2] = np.moveaxis(nat, -1, 0)
    return out


def from_padded(p: np.ndarray) -> np.ndarray:
    """padded SoA -> natural AoS (mz,my,mx,nc)."""
    return np.ascontiguousarray(np.moveaxis(p[:, 2:-2, 2:-2, 2:-2], 0, -1))


def local_to_padded(cfg: Config, loc: np.ndarray, nc: int) -> np.ndarray:
    """PETSc ghosted local Vec (periodic in every direction) -> padded SoA."""
    loc = np.asarray(loc).reshape(cfg.mz + 4, cfg.my + 4, cfg.mx + 4, nc)
    return np.ascontiguousarray(np.moveaxis(loc, -1, 0))


def _ptrs(planes):
    arr = (C.POINTER(C.c_double) * len(planes))()
    for a, pl in enumerate(planes):
        assert pl.dtype == np.float64 and pl.flags.c_contiguous
        arr[a] = pl.ctypes.data_as(C.POINTER(C.c_double))
    return arr


def _dp(a: Optional[np.ndarray]):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


# ------------------------------------------------------------ restatement --
def build_oracle(force: bool = False) -> str:
    """Compile the C restatement (committed sources) if its .so is missing."""
    if force or not os.path.exists(ORACLE_SO):
        subprocess.run(["make", "-s", "-C", _HERE, "_build/liboracle.so"], check=True)
    return ORACLE_SO


def build_oracle_count(force: bool = False) -> str:
    """Compile the operation-counting build of the restatement if missing."""
    if force or not os.path.exists(ORACLE_COUNT_SO):
        subprocess.run(["make", "-s", "-C", _HERE, "_build/liboracle_count.so"], check=True)
    return ORACLE_COUNT_SO


class Oracle:
    """ctypes front end of oracle/src/cb_oracle.c (padded SoA numpy arrays).

    counting=True loads the operation-counting build of the same source
    (identical results; ``count_reset`` / ``count_read`` give the number of
    floating-point operations by kind since the last reset)."""

    COUNT_KINDS = ("add", "mul", "div", "sqrt", "pow", "cmp", "abs")

    def __init__(self, cfg: Config, counting: bool = False):
        self.cfg = cfg
        self.lib = C.CDLL(build_oracle_count() if counting else build_oracle())
        self.counting = counting
        self.c = _ccfg(cfg)
        PP = C.POINTER(C.POINTER(C.c_double))
        D = C.POINTER(C.c_double)
        L = self.lib
        L.cbo_fill_ghosts.argtypes = [C.c_void_p, D]
        L.cbo_weno5.argtypes = [C.c_double] * 5
        L.cbo_weno5.restype = C.c_double
        L.cbo_metrics.argtypes = [C.c_void_p, PP, PP, PP, PP, D]
        L.cbo_eos.argtypes = [C.c_void_p, PP, D]
        L.cbo_sigma.argtypes = [C.c_void_p, PP]
        L.cbo_sigma_sensor.argtypes = [C.c_void_p, PP, PP]
        L.cbo_rhs.argtypes = [C.c_void_p, PP, PP, PP, PP, D, D, D, PP, PP]
        L.cbo_rhs.restype = C.c_int
        L.cbo_eddy_viscosity.argtypes = [C.c_void_p, PP, PP, PP, PP, D, D, D]
        L.cbo_steps.argtypes = [C.c_void_p, C.c_int, PP, PP, PP, C.POINTER(C.c_int), D, PP, PP, PP, D, D]
        L.cbo_steps.restype = C.c_int
        L.cbo_bc_periodic.argtypes = [C.c_void_p, PP, PP]
        L.cbo_bc_periodic.restype = C.c_int
        L.cbo_formbcs.argtypes = [C.c_void_p, C.c_double, PP, PP, PP, PP, D, D, PP]
        L.cbo_formbcs.restype = C.c_int
        L.cbo_ibm_interpolate.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, PP, PP, D, PP, C.c_int,
                                          C.c_int, C.c_int, D]
        L.cbo_ibm_interpolate.restype = C.c_int
        L.cbo_steps_ibm.argtypes = [C.c_void_p, C.c_int, PP, PP, PP, C.POINTER(C.c_int), D, PP, PP, PP, D, D,
                                    C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, PP, D, C.POINTER(C.c_int),
                                    C.c_int, C.c_int]
        L.cbo_steps_ibm.restype = C.c_int
        L.cbo_dynamic_smagorinsky.argtypes = [C.c_void_p, PP, PP, D, PP, PP, PP, D, D, D]
        L.cbo_dynamic_smagorinsky.restype = C.c_int
        L.cbo_eddy_viscosity_dyn.argtypes = [C.c_void_p, PP, PP, PP, PP, PP, D, D, D, D]
        self._cp = C.byref(self.c)

    def set_coordinates(self, coor_pad: np.ndarray) -> None:
        """Node coordinates (3, padded) for the boundary codes that read them
        (k-lo inflow 52 and 47)."""
        self._coor = np.ascontiguousarray(coor_pad, dtype=np.float64)
        self.c.coor_x = self._coor[0].ctypes.data
        self.c.coor_y = self._coor[1].ctypes.data

    def count_reset(self) -> None:
        self.lib.cbo_count_reset()

    def count_read(self) -> dict:
        buf = (C.c_longlong * len(self.COUNT_KINDS))()
        self.lib.cbo_count_read(buf)
        return dict(zip(self.COUNT_KINDS, (int(v) for v in buf)))

    def weno5(self, a: float, b: float, c: float, d: float, e: float) -> float:
        """WENO5-JS value at x_{i+1/2} from v_{i-2..i+2} (left-biased)."""
        return float(self.lib.cbo_weno5(a, b, c, d, e))

    def zeros(self, nc: int) -> np.ndarray:
        return np.zeros((nc,) + self.cfg.padded_shape)

    def fill_ghosts(self, f: np.ndarray) -> np.ndarray:
        for a in range(f.shape[0]):
            self.lib.cbo_fill_ghosts(self._cp, _dp(f[a]))
        return f

    def metrics(self, coor_pad: np.ndarray):
        """coor_pad: (3, padded) -> dict csi/eta/zet (3, padded), aj (1, padded)."""
        csi, eta, zet, aj = self.zeros(3), self.zeros(3), self.zeros(3), self.zeros(1)
        self.lib.cbo_metrics(self._cp, _ptrs(list(coor_pad)), _ptrs(list(csi)), _ptrs(list(eta)),
                             _ptrs(list(zet)), _dp(aj[0]))
        return {"csi": csi, "eta": eta, "zet": zet, "aj": aj}

    def eos(self, q: np.ndarray) -> np.ndarray:
        p = self.zeros(1)
        self.lib.cbo_eos(self._cp, _ptrs(list(q)), _dp(p[0]))
        return p

    def sigma(self, q: Optional[np.ndarray] = None) -> np.ndarray:
        """Hybrid weights at istage 0: constant (sensor off) or from the ghosted
        stage state q with -calc_sigma 1."""
        s = self.zeros(3)
        if self.cfg.calc_sigma:
            if q is None:
                raise ValueError("the shock sensor needs the stage state")
            self.lib.cbo_sigma_sensor(self._cp, _ptrs(list(q)), _ptrs(list(s)))
        else:
            self.lib.cbo_sigma(self._cp, _ptrs(list(s)))
        return s

    def eddy_viscosity(self, qu: Optional[np.ndarray], met, nvert: np.ndarray, nut: np.ndarray):
        self.lib.cbo_eddy_viscosity(self._cp, _ptrs(list(qu)) if qu is not None else None,
                                    _ptrs(list(met["csi"])), _ptrs(list(met["eta"])),
                                    _ptrs(list(met["zet"])), _dp(met["aj"][0]), _dp(nvert[0]),
                                    _dp(nut[0]))
        return nut

    def rhs(self, q: np.ndarray, met, nvert: np.ndarray, nut: Optional[np.ndarray] = None,
            sig: Optional[np.ndarray] = None) -> np.ndarray:
        out = self.zeros(5)
        e = self.lib.cbo_rhs(self._cp, _ptrs(list(q)), _ptrs(list(met["csi"])), _ptrs(list(met["eta"])),
                             _ptrs(list(met["zet"])), _dp(met["aj"][0]), _dp(nvert[0]),
                             _dp(nut[0]) if nut is not None else None,
                             _ptrs(list(sig)) if sig is not None else None, _ptrs(list(out)))
        if e:
            raise RuntimeError(f"cbo_rhs failed with status {e}")
        return out

    def steps(self, nsteps: int, state: dict, met, nvert: np.ndarray) -> dict:
        """state: dict q, qold, quc (padded 5), have_uc (int), nut (padded 1); updated in place."""
        hu = C.c_int(int(state["have_uc"]))
        e = self.lib.cbo_steps(self._cp, nsteps, _ptrs(list(state["q"])), _ptrs(list(state["qold"])),
                               _ptrs(list(state["quc"])), C.byref(hu), _dp(state["nut"][0]),
                               _ptrs(list(met["csi"])), _ptrs(list(met["eta"])), _ptrs(list(met["zet"])),
                               _dp(met["aj"][0]), _dp(nvert[0]))
        if e:
            raise RuntimeError(f"cbo_steps failed with status {e}")
        state["have_uc"] = hu.value
        return state

    def initial_state(self, q_nat: np.ndarray) -> dict:
        q = self.fill_ghosts(to_padded(self.cfg, q_nat))
        return {"q": q, "qold": q.copy(), "quc": np.zeros_like(q), "have_uc": 0, "nut": self.zeros(1)}

    def dynamic_smagorinsky(self, q: np.ndarray, quc: Optional[np.ndarray], met, nvert: np.ndarray,
                            cs: Optional[np.ndarray] = None, lp: Optional[np.ndarray] = None) -> np.ndarray:
        """Compute_Smagorinsky_Constant_1 with -les 2: Cs (padded 1) from the
        ghosted state q and the last CalcUCat state quc (None: zero velocity);
        lp defaults to the EqOfState of q."""
        cs = self.zeros(1) if cs is None else cs
        lp = self.eos(q) if lp is None else lp
        e = self.lib.cbo_dynamic_smagorinsky(self._cp, _ptrs(list(q)), _ptrs(list(quc)) if quc is not None else None,
                                             _dp(lp[0]), _ptrs(list(met["csi"])), _ptrs(list(met["eta"])),
                                             _ptrs(list(met["zet"])), _dp(met["aj"][0]), _dp(nvert[0]), _dp(cs[0]))
        if e:
            raise RuntimeError(f"cbo_dynamic_smagorinsky failed with status {e}")
        return cs

    def eddy_viscosity_dyn(self, q: np.ndarray, quc: Optional[np.ndarray], met, nvert: np.ndarray, cs: np.ndarray,
                           nut: np.ndarray) -> np.ndarray:
        self.lib.cbo_eddy_viscosity_dyn(self._cp, _ptrs(list(q)), _ptrs(list(quc)) if quc is not None else None,
                                        _ptrs(list(met["csi"])), _ptrs(list(met["eta"])), _ptrs(list(met["zet"])),
                                        _dp(met["aj"][0]), _dp(nvert[0]), _dp(cs[0]), _dp(nut[0]))
        return nut

    def formbcs(self, alfa: float, lq: np.ndarray, qold: np.ndarray, met, q: np.ndarray,
                nvert: Optional[np.ndarray] = None) -> np.ndarray:
        """FormBCS(user, alfa) on q (padded 5, in/out) from the ghosted lq."""
        e = self.lib.cbo_formbcs(self._cp, alfa, _ptrs(list(lq)), _ptrs(list(qold)), _ptrs(list(met["eta"])),
                                 _ptrs(list(met["zet"])), _dp(met["aj"][0]),
                                 _dp(nvert[0]) if nvert is not None else None, _ptrs(list(q)))
        if e:
            raise RuntimeError(f"cbo_formbcs failed with status {e}")
        return q

    def ibm_interpolate(self, surface: "IbmSurface", info: np.ndarray, coor_pad: np.ndarray, q: np.ndarray,
                        p: np.ndarray, add_dundt: int = 1, ustar: Optional[np.ndarray] = None,
                        qold: Optional[np.ndarray] = None) -> None:
        """ibm_interpolation_advanced on q (padded 5) and p (padded 1), in
        place; with -wallfunction 2, ustar (one double per list entry) receives
        u_tau of the last sweep; qold (padded 5): the state whose density the
        -isothermal 2 wall reads (default: q as given)."""
        info = np.ascontiguousarray(info, dtype=IBM_INFO_DTYPE)
        if ustar is not None:
            assert ustar.dtype == np.float64 and ustar.size >= info.size and ustar.flags.c_contiguous
        e = self.lib.cbo_ibm_interpolate(self._cp, C.byref(surface.c), info.size, info.ctypes.data,
                                         _ptrs(list(coor_pad)), _ptrs(list(q)), _dp(p[0]),
                                         _ptrs(list(qold)) if qold is not None else None, add_dundt,
                                         self.cfg.twoD, self.cfg.wallfunction,
                                         _dp(ustar) if ustar is not None else None)
        if e:
            raise RuntimeError(f"cbo_ibm_interpolate failed with status {e}")

    def steps_immersed(self, nsteps: int, state: dict, met, nvert: np.ndarray, surface, info,
                       coor_pad: np.ndarray) -> dict:
        """Time steps with immersed bodies (cbo_steps_ibm): surface / info are
        one body's IbmSurface and list, or equal-length sequences of them.
        state as for steps() plus "lp" (padded 1: the pressure the reference
        carries in P / lP) and "lp_valid", both updated in place."""
        surfs = list(surface) if isinstance(surface, (list, tuple)) else [surface]
        infos = list(info) if isinstance(info, (list, tuple)) else [info]
        infos = [np.ascontiguousarray(a, dtype=IBM_INFO_DTYPE) for a in infos]
        nb = len(surfs)
        sarr = (_CSurf * nb)(*[s.c for s in surfs])
        nl = (C.c_int * nb)(*[a.size for a in infos])
        lp = (C.c_void_p * nb)(*[a.ctypes.data for a in infos])
        if "lp" not in state:
            state["lp"] = self.zeros(1)
            state["lp_valid"] = 0
        hu = C.c_int(int(state["have_uc"]))
        lv = C.c_int(int(state["lp_valid"]))
        e = self.lib.cbo_steps_ibm(self._cp, nsteps, _ptrs(list(state["q"])), _ptrs(list(state["qold"])),
                                   _ptrs(list(state["quc"])), C.byref(hu), _dp(state["nut"][0]),
                                   _ptrs(list(met["csi"])), _ptrs(list(met["eta"])), _ptrs(list(met["zet"])),
                                   _dp(met["aj"][0]), _dp(nvert[0]), nb, sarr, nl, lp, _ptrs(list(coor_pad)),
                                   _dp(state["lp"][0]), C.byref(lv), self.cfg.twoD, self.cfg.wallfunction)
        if e:
            raise RuntimeError(f"cbo_steps_ibm failed with status {e}")
        state["have_uc"] = hu.value
        state["lp_valid"] = lv.value
        return state


# ------------------------------------------------------ immersed boundary --
# One entry of the interpolation list: cbo_ibm_info (oracle/src/cb_oracle.h),
# the IBMInfo fields the interpolation reads (variables.h:50-89).
IBM_INFO_DTYPE = np.dtype([
    ("ni", "<i4"), ("nj", "<i4"), ("nk", "<i4"), ("cell", "<i4"),
    ("i1", "<i4"), ("j1", "<i4"), ("k1", "<i4"), ("i2", "<i4"), ("j2", "<i4"), ("k2", "<i4"),
    ("i3", "<i4"), ("j3", "<i4"), ("k3", "<i4"), ("pad", "<i4"),
    ("cr1", "<f8"), ("cr2", "<f8"), ("cr3", "<f8"), ("cs1", "<f8"), ("cs2", "<f8"), ("cs3", "<f8"),
    ("d_s", "<f8"), ("d_i", "<f8"), ("pmin", "<f8", (3,)),
])
_IBM_INTS = ("ni", "nj", "nk", "cell", "i1", "j1", "k1", "i2", "j2", "k2", "i3", "j3", "k3")
_IBM_REALS = ("cr1", "cr2", "cr3", "cs1", "cs2", "cs3", "d_s", "d_i")


def ibm_info_from_flat(iv: np.ndarray, rv: np.ndarray) -> np.ndarray:
    """13 ints + 11 doubles per entry (the reference driver's layout) -> list."""
    n = iv.size // 13
    iv, rv = iv.reshape(n, 13), rv.reshape(n, 11)
    out = np.zeros(n, dtype=IBM_INFO_DTYPE)
    for a, f in enumerate(_IBM_INTS):
        out[f] = iv[:, a]
    for a, f in enumerate(_IBM_REALS):
        out[f] = rv[:, a]
    out["pmin"] = rv[:, 8:11]
    return out


def ibm_info_to_flat(info: np.ndarray):
    iv = np.stack([info[f] for f in _IBM_INTS], axis=1).astype(np.int32)
    rv = np.concatenate([np.stack([info[f] for f in _IBM_REALS], axis=1), info["pmin"]], axis=1)
    return np.ascontiguousarray(iv), np.ascontiguousarray(rv, dtype=np.float64)


class _CSurf(C.Structure):
    _fields_ = [("n_v", C.c_int), ("n_elmt", C.c_int), ("nv1", C.c_void_p), ("nv2", C.c_void_p),
                ("nv3", C.c_void_p), ("nf_x", C.c_void_p), ("nf_y", C.c_void_p), ("nf_z", C.c_void_p),
                ("u", C.c_void_p), ("uold", C.c_void_p)]


class IbmSurface:
    """cbo_ibm_surface over numpy arrays (kept alive here): a dict with x, y, z,
    nv1..nv3, nf_x..nf_z (workloads.sphere_surface) and vertex velocities
    u, uold of shape (n_v, 3) (zero when absent)."""

    def __init__(self, s: dict, u: Optional[np.ndarray] = None, uold: Optional[np.ndarray] = None):
        self.a = {k: np.ascontiguousarray(s[k], dtype=np.int32) for k in ("nv1", "nv2", "nv3")}
        self.a.update({k: np.ascontiguousarray(s[k], dtype=np.float64) for k in ("nf_x", "nf_y", "nf_z")})
        n_v = len(s["x"])
        self.a["u"] = np.ascontiguousarray(np.zeros((n_v, 3)) if u is None else u, dtype=np.float64)
        self.a["uold"] = np.ascontiguousarray(np.zeros((n_v, 3)) if uold is None else uold, dtype=np.float64)
        c = _CSurf()
        c.n_v, c.n_elmt = n_v, len(s["nv1"])
        for k, v in self.a.items():
            setattr(c, k, v.ctypes.data)
        self.c = c


# ------------------------------------------------------ shim-built reference --
def ref_available() -> bool:
    return os.path.exists(REF_SO) or os.path.isdir(REF_SRC_DIR)


def build_ref(force: bool = False, optimized: bool = False, io: bool = False) -> str:
    so = REF_IO_SO if io else (REF_SO_O3 if optimized else REF_SO)
    if force or not os.path.exists(so):
        if not os.path.isdir(REF_SRC_DIR):
            raise FileNotFoundError("reference sources not present; cannot build oracle/_ref")
        subprocess.run(["make", "-s", "-C", _HERE, "ref", f"REF_DIR={REF_SRC_DIR}"], check=True)
    return so


class RefOracle:
    """The reference's own hot-path C (via the PETSc shim); one live instance
    per process (the reference keeps its state in globals)."""

    def __init__(self, cfg: Config, coords_nat: np.ndarray, optimized: bool = False, io: bool = False):
        if cfg.flux != 0:
            raise ValueError("the reference has no Roe flux (flux 1); check it against the restatement")
        if cfg.weno_order != 3:
            raise ValueError("the reference has no WENO5 (weno_order 5); check it against the restatement")
        self.cfg = cfg
        self.lib = C.CDLL(build_ref(optimized=optimized, io=io))
        self.io = io
        L = self.lib
        D = C.POINTER(C.c_double)
        L.ref_setup.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int), D, C.c_char_p]
        for f in ("ref_set_nvert", "ref_set_state", "ref_set_local_state", "ref_set_nut", "ref_get_Q",
                  "ref_get_P", "ref_get_lQ", "ref_get_lP", "ref_get_nut", "ref_get_lnut",
                  "ref_get_lsigma", "ref_get_lucat"):
            getattr(L, f).argtypes = [D]
        L.ref_rhs.argtypes = [C.c_int, D]
        L.ref_steps.argtypes = [C.c_int]
        L.ref_get_metrics.argtypes = [D, D, D, D]
        coords = np.ascontiguousarray(coords_nat, dtype=np.float64)
        assert coords.shape == (cfg.mz, cfg.my, cfg.mx, 3)
        bc = (C.c_int * 6)(*cfg.bctype)
        e = L.ref_setup(cfg.mx, cfg.my, cfg.mz, bc, _dp(coords), cfg.ref_options().encode())
        if e:
            raise RuntimeError(f"ref_setup failed ({e})")
        self.nnodes = cfg.mx * cfg.my * cfg.mz
        gx, gy, gz = C.c_int(), C.c_int(), C.c_int()
        L.ref_local_dims(C.byref(gx), C.byref(gy), C.byref(gz))
        self.ldims = (gz.value, gy.value, gx.value)

    def set_nvert(self, nvert_nat: np.ndarray):
        a = np.ascontiguousarray(nvert_nat, dtype=np.float64).reshape(-1)
        assert a.size == self.nnodes
        self.lib.ref_set_nvert(_dp(a))

    def write_checkpoint(self, ti: int) -> None:
        """The reference's Q_P_Binary_Output (main.c:247-304) as time step ti,
        block 0, into the working directory (needs io=True)."""
        if not self.io or self.lib.ref_write_checkpoint(ti):
            raise RuntimeError("Q_P_Binary_Output failed")

    def restart(self, ti: int) -> None:
        """The reference's RestartApplication (main.c:620-693) from the files
        of time step ti in the working directory (needs io=True)."""
        if not self.io or self.lib.ref_restart(ti):
            raise RuntimeError("RestartApplication failed")

    def set_state(self, q_nat: np.ndarray):
        a = np.ascontiguousarray(q_nat, dtype=np.float64).reshape(-1)
        assert a.size == 5 * self.nnodes
        self.lib.ref_set_state(_dp(a))

    def calc_ucat(self):
        return self.lib.ref_calc_ucat()

    def eddy_viscosity(self):
        return self.lib.ref_eddy_viscosity()

    def rhs(self, istage: int = 0) -> np.ndarray:
        out = np.zeros(5 * self.nnodes)
        e = self.lib.ref_rhs(istage, _dp(out))
        if e:
            raise RuntimeError(f"ref_rhs failed ({e})")
        return out.reshape(self.cfg.mz, self.cfg.my, self.cfg.mx, 5)

    def steps(self, n: int):
        return self.lib.ref_steps(n)

    def Q(self) -> np.ndarray:
        out = np.zeros(5 * self.nnodes)
        self.lib.ref_get_Q(_dp(out))
        return out.reshape(self.cfg.mz, self.cfg.my, self.cfg.mx, 5)

    def P(self) -> np.ndarray:
        out = np.zeros(self.nnodes)
        self.lib.ref_get_P(_dp(out))
        return out.reshape(self.cfg.mz, self.cfg.my, self.cfg.mx)

    def nut(self) -> np.ndarray:
        out = np.zeros(self.nnodes)
        self.lib.ref_get_nut(_dp(out))
        return out.reshape(self.cfg.mz, self.cfg.my, self.cfg.mx)

    def cs(self) -> np.ndarray:
        out = np.zeros(self.nnodes)
        self.lib.ref_get_cs(_dp(out))
        return out.reshape(self.cfg.mz, self.cfg.my, self.cfg.mx)

    def local(self, which: str, nc: int) -> np.ndarray:
        gz, gy, gx = self.ldims
        out = np.zeros(gz * gy * gx * nc)
        getattr(self.lib, f"ref_get_{which}")(_dp(out))
        return out.reshape(gz, gy, gx, nc)

    def ibm_setup(self, s: dict):
        """One immersed body (ibi 0) from a surface dict (workloads.sphere_surface)."""
        L = self.lib
        self._surf = {k: np.ascontiguousarray(s[k], dtype=np.float64) for k in ("x", "y", "z", "nf_x", "nf_y", "nf_z")}
        self._surf.update({k: np.ascontiguousarray(s[k], dtype=np.int32) for k in ("nv1", "nv2", "nv3")})
        a = self._surf
        e = L.ref_ibm_setup(len(a["x"]), len(a["nv1"]), *(C.c_void_p(a[k].ctypes.data) for k in (
            "x", "y", "z", "nv1", "nv2", "nv3", "nf_x", "nf_y", "nf_z")))
        if e:
            raise RuntimeError(f"ref_ibm_setup failed ({e})")

    def ibm_set_velocity(self, u: np.ndarray, uold: np.ndarray):
        u = np.ascontiguousarray(u, dtype=np.float64)
        uold = np.ascontiguousarray(uold, dtype=np.float64)
        self.lib.ref_ibm_set_velocity(C.c_void_p(u.ctypes.data), C.c_void_p(uold.ctypes.data))

    def ibm_search(self):
        """ibm_search_advanced: returns (nvert natural, interpolation list)."""
        L = self.lib
        if L.ref_ibm_search():
            raise RuntimeError("ref_ibm_search failed")
        nv = np.zeros(self.nnodes)
        L.ref_get_nvert(_dp(nv))
        return nv.reshape(self.cfg.mz, self.cfg.my, self.cfg.mx), self.ibm_list()

    def ibm_list(self) -> np.ndarray:
        L = self.lib
        n = L.ref_ibm_list_count()
        iv, rv = np.zeros(13 * n, dtype=np.int32), np.zeros(11 * n)
        L.ref_ibm_list_get(C.c_void_p(iv.ctypes.data), C.c_void_p(rv.ctypes.data))
        return ibm_info_from_flat(iv, rv)

    def ibm_set_list(self, info: np.ndarray):
        iv, rv = ibm_info_to_flat(info)
        self.lib.ref_ibm_list_set(info.size, C.c_void_p(iv.ctypes.data), C.c_void_p(rv.ctypes.data))

    def ibm_interpolate(self, add_dundt: int = 1):
        if self.lib.ref_ibm_interpolate(add_dundt):
            raise RuntimeError("ref_ibm_interpolate failed")

    def formbcs(self, alfa: float):
        self.lib.ref_formbcs.argtypes = [C.c_double]
        return self.lib.ref_formbcs(alfa)

    def metrics_local(self):
        gz, gy, gx = self.ldims
        n = gz * gy * gx
        csi, eta, zet, aj = np.zeros(3 * n), np.zeros(3 * n), np.zeros(3 * n), np.zeros(n)
        self.lib.ref_get_metrics(_dp(csi), _dp(eta), _dp(zet), _dp(aj))
        sh = (gz, gy, gx)
        return {"csi": csi.reshape(sh + (3,)), "eta": eta.reshape(sh + (3,)),
                "zet": zet.reshape(sh + (3,)), "aj": aj.reshape(sh + (1,))}


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    """Relative L2 of a against the reference b (0 if both are zero)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = float(np.linalg.norm(b))
    d = float(np.linalg.norm(a - b))
    if nb == 0.0:
        return d
    return d / nb
