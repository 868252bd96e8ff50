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
REF_SO = os.path.join(_HERE, "_ref", "libchimera_ref.so")
REF_SO_O3 = os.path.join(_HERE, "_ref", "libchimera_ref_O3.so")
REF_SRC_DIR = os.environ.get("CHIMERA_REF_DIR", "/root/reference")


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

    def ref_options(self) -> str:
        o = [
            ("-les", self.les), ("-inv", self.inviscid), ("-fluxorder", self.fluxorder),
            ("-ENOorder", self.eno_order), ("-central", self.central),
            ("-isothermal", self.isothermal), ("-s_x", repr(float(self.s_x))),
            ("-s_y", repr(float(self.s_y))), ("-s_z", repr(float(self.s_z))),
            ("-ren", repr(float(self.ren))), ("-Ma", repr(float(self.ma))),
            ("-Pr", repr(float(self.pr))), ("-gamma", repr(float(self.gamma))),
            ("-dt", repr(float(self.dt))), ("-visT", 0), ("-twoD", 0), ("-TwoD", 0),
            ("-calc_sigma", self.calc_sigma), ("-s_x_min", repr(float(self.s_x_min))),
            ("-s_y_min", repr(float(self.s_y_min))), ("-s_z_min", repr(float(self.s_z_min))),
            ("-sigma_thrsh", repr(float(self.sigma_thrsh))),
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
        ("flux", C.c_int),
    ]


def _ccfg(cfg: Config) -> _CCfg:
    c = _CCfg()
    for f, _ in _CCfg._fields_:
        if f == "bctype":
            c.bctype = (C.c_int * 6)(*cfg.bctype)
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


class Oracle:
    """ctypes front end of oracle/src/cb_oracle.c (padded SoA numpy arrays)."""

    def __init__(self, cfg: Config):
        self.cfg = cfg
        self.lib = C.CDLL(build_oracle())
        self.c = _ccfg(cfg)
        PP = C.POINTER(C.POINTER(C.c_double))
        D = C.POINTER(C.c_double)
        L = self.lib
        L.cbo_fill_ghosts.argtypes = [C.c_void_p, D]
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
        self._cp = C.byref(self.c)

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


# ------------------------------------------------------ shim-built reference --
def ref_available() -> bool:
    return os.path.exists(REF_SO) or os.path.isdir(REF_SRC_DIR)


def build_ref(force: bool = False, optimized: bool = False) -> str:
    so = REF_SO_O3 if optimized else REF_SO
    if force or not os.path.exists(so):
        if not os.path.isdir(REF_SRC_DIR):
            raise FileNotFoundError("reference sources not present; cannot build oracle/_ref")
        subprocess.run(["make", "-s", "-C", _HERE, "ref", f"REF_DIR={REF_SRC_DIR}"], check=True)
    return so


class RefOracle:
    """The reference's own hot-path C (via the PETSc shim); one live instance
    per process (the reference keeps its state in globals)."""

    def __init__(self, cfg: Config, coords_nat: np.ndarray, optimized: bool = False):
        if cfg.flux != 0:
            raise ValueError("the reference has no Roe flux (flux 1); check it against the restatement")
        self.cfg = cfg
        self.lib = C.CDLL(build_ref(optimized=optimized))
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

    def local(self, which: str, nc: int) -> np.ndarray:
        gz, gy, gx = self.ldims
        out = np.zeros(gz * gy * gx * nc)
        getattr(self.lib, f"ref_get_{which}")(_dp(out))
        return out.reshape(gz, gy, gx, nc)

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
