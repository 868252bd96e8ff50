"""Batched multi-block form over the C-ABI (cb_batch_* in include/chimera_b200.h).

The reference advances its blocks one after another inside the time step
(solvers.c:246, ``for (bi = 0; bi < block_number; bi++)`` around RungeKutta),
each with its own FormBCS (rhs.c:1107-1227) and DMGlobalToLocal.  ``Batch``
keeps every block resident on one GPU and advances all of them with one
persistent stage launch per RK stage; the boundary and ghost nodes of all
blocks are then filled by one gather from a halo map.

Halo maps are int32 arrays of shape (n, 9): (dst block, di, dj, dk, src block,
si, sj, sk, from_stage_input), node indices -2..m+1 in each block's own
(i, j, k).  Three generators are provided:

  halo_maps_self_periodic(dims)      each block wraps onto itself: the
                                     single-block periodic path, block by block
  halo_maps_decomposed(gdims, parts) sub-blocks of one periodic box: the
                                     batch reproduces the undivided box
  halo_maps_donor(dims, perm)        every block's 2-node halo taken from the
                                     interior of a donor block (perm[b])

Each returns (stage_map, wrap_map): the stage map is applied after every RK
stage, the wrap map (plain DMGlobalToLocal, sources never destinations) to the
eddy viscosity each step and once to the uploaded state.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Sequence, Tuple

import numpy as np

from . import _lib
from ._lib import CbConfig, ChimeraError, dptr

HALO_STAGE, HALO_WRAP = 0, 1


# ------------------------------------------------------------ halo maps --
def _padded_nodes(dims):
    """All padded nodes (i, j, k), -2..m+1, of a block, and the non-interior mask."""
    mx, my, mz = dims
    k, j, i = np.meshgrid(np.arange(-2, mz + 2), np.arange(-2, my + 2), np.arange(-2, mx + 2), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    inter = (i >= 1) & (i <= mx - 2) & (j >= 1) & (j <= my - 2) & (k >= 1) & (k <= mz - 2)
    return i, j, k, ~inter


def _wrap(x, m):
    return np.where(x < 0, x + m, np.where(x >= m, x - m, x))


def _stage_source(gi, gj, gk, M):
    """Single-block periodic FormBCS + DMGlobalToLocal rule for non-interior
    nodes (rhs.c:1107-1227): the owned image oi = wrap(i); if that image is an
    interior node its stage output is taken, otherwise the stale stage input
    two nodes across the face, with k faces winning over j over i."""
    MX, MY, MZ = M
    oi, oj, ok = _wrap(gi, MX), _wrap(gj, MY), _wrap(gk, MZ)
    si, sj, sk = oi.copy(), oj.copy(), ok.copy()
    bnd = (oi == 0) | (oi == MX - 1) | (oj == 0) | (oj == MY - 1) | (ok == 0) | (ok == MZ - 1)
    c_k0 = bnd & (ok == 0)
    c_k1 = bnd & ~c_k0 & (ok == MZ - 1)
    rest = bnd & ~c_k0 & ~c_k1
    c_j0 = rest & (oj == 0)
    c_j1 = rest & ~c_j0 & (oj == MY - 1)
    rest = rest & ~c_j0 & ~c_j1
    c_i0 = rest & (oi == 0)
    c_i1 = rest & ~c_i0
    sk = np.where(c_k0, ok - 2, np.where(c_k1, ok + 2, sk))
    sj = np.where(c_j0, oj - 2, np.where(c_j1, oj + 2, sj))
    si = np.where(c_i0, oi - 2, np.where(c_i1, oi + 2, si))
    return si, sj, sk, bnd.astype(np.int32)


def halo_maps_self_periodic(dims: Sequence[Tuple[int, int, int]], coded: Sequence[int] = ()):
    """Every block periodic on its own: the single-block path, block by block.
    Blocks listed in `coded` (given face codes with Batch.set_bctype, which run
    their own FormBCS) get no entries, as cb_batch_halo_periodic leaves them."""
    st, wr = [], []
    skip = set(int(b) for b in coded)
    for b, d in enumerate(dims):
        if b in skip:
            continue
        i, j, k, non = _padded_nodes(d)
        i, j, k = i[non], j[non], k[non]
        si, sj, sk, fin = _stage_source(i, j, k, d)
        bb = np.full_like(i, b)
        st.append(np.stack([bb, i, j, k, bb, si, sj, sk, fin], axis=1))
        oi, oj, ok = _wrap(i, d[0]), _wrap(j, d[1]), _wrap(k, d[2])
        g = (oi != i) | (oj != j) | (ok != k)
        wr.append(np.stack([bb[g], i[g], j[g], k[g], bb[g], oi[g], oj[g], ok[g], np.zeros_like(i[g])], axis=1))
    return (np.ascontiguousarray(np.concatenate(st).astype(np.int32)),
            np.ascontiguousarray(np.concatenate(wr).astype(np.int32)))


def decompose(gdims: Tuple[int, int, int], cuts: Sequence[Sequence[int]]):
    """Sub-blocks of a periodic box of gdims nodes (interior 1..M-2 per
    direction).  cuts[d] lists the interior sizes along direction d (summing
    to M-2).  Returns [(offset (i0, j0, k0), dims (mx, my, mz))]: local node l
    is global node l + offset, local 0..m-1 covers the sub-block's interior
    plus one boundary node on each side."""
    for d in range(3):
        if sum(cuts[d]) != gdims[d] - 2 or min(cuts[d]) < 4:
            raise ValueError("cuts must cover the interior, each part >= 4 nodes")
    parts = []
    starts = [np.concatenate([[0], np.cumsum(c)[:-1]]) for c in cuts]
    for kz, nz in zip(starts[2], cuts[2]):
        for jy, ny in zip(starts[1], cuts[1]):
            for ix, nx in zip(starts[0], cuts[0]):
                parts.append(((int(ix), int(jy), int(kz)), (int(nx) + 2, int(ny) + 2, int(nz) + 2)))
    return parts


def halo_maps_decomposed(gdims: Tuple[int, int, int], parts, only=None):
    """Maps under which the sub-blocks `parts` (from ``decompose``) evolve as
    the undivided periodic box: every non-interior node takes what the
    single-block rule gives at its global position, read from the block that
    owns the source node as interior (stage output), or, for a stale-input
    source (a global ghost node), from the block owning the nearest interior
    node, in whose padded box it lies.  `only`: destination blocks to list
    (default all) -- a process needs its own blocks and their neighbours."""
    M = np.array(gdims)
    offs = np.array([p[0] for p in parts])
    dims = np.array([p[1] for p in parts])
    # owner lookup of a global interior node per direction
    owner_axis = []
    for d in range(3):
        starts = sorted(set(int(o[d]) for o in offs))
        owner_axis.append(np.array(starts))

    def owner(gi, gj, gk):
        g = np.stack([gi, gj, gk], axis=1)
        g = np.clip(g, 1, M - 2)
        idx = np.zeros(len(gi), dtype=np.int64)
        # block index from the per-direction slab indices (parts are ordered x fastest)
        n = [len(a) for a in owner_axis]
        slab = [np.searchsorted(owner_axis[d], g[:, d] - 1, side="right") - 1 for d in range(3)]
        idx = (slab[2] * n[1] + slab[1]) * n[0] + slab[0]
        return idx

    st, wr = [], []
    for b, (off, d) in enumerate(parts):
        if only is not None and b not in only:
            continue
        i, j, k, non = _padded_nodes(d)
        i, j, k = i[non], j[non], k[non]
        gi, gj, gk = i + off[0], j + off[1], k + off[2]
        si, sj, sk, fin = _stage_source(gi, gj, gk, gdims)
        ob = owner(si, sj, sk)
        bb = np.full_like(i, b)
        st.append(np.stack([bb, i, j, k, ob, si - offs[ob, 0], sj - offs[ob, 1], sk - offs[ob, 2], fin], axis=1))
        # wrap map
        oi, oj, ok = _wrap(gi, M[0]), _wrap(gj, M[1]), _wrap(gk, M[2])
        img_int = (oi >= 1) & (oi <= M[0] - 2) & (oj >= 1) & (oj <= M[1] - 2) & (ok >= 1) & (ok <= M[2] - 2)
        owned = (i >= 0) & (i <= d[0] - 1) & (j >= 0) & (j <= d[1] - 1) & (k >= 0) & (k <= d[2] - 1)
        g = img_int | ~owned
        ob = owner(oi[g], oj[g], ok[g])
        wr.append(np.stack([bb[g], i[g], j[g], k[g], ob, oi[g] - offs[ob, 0], oj[g] - offs[ob, 1], ok[g] - offs[ob, 2],
                            np.zeros_like(i[g])], axis=1))
    return (np.ascontiguousarray(np.concatenate(st).astype(np.int32)),
            np.ascontiguousarray(np.concatenate(wr).astype(np.int32)))


def halo_maps_donor(dims: Sequence[Tuple[int, int, int]], perm: Sequence[int]):
    """2-node overlap halo of every block taken from the interior of the donor
    block perm[b]: a node below a face reads the donor's last interior nodes,
    a node above it the donor's first ones, and tangential indices wrap into the
    donor's interior.  Sources are interior, read from the stage output."""
    st = []
    for b, d in enumerate(dims):
        dn = dims[perm[b]]
        i, j, k, non = _padded_nodes(d)
        i, j, k = i[non], j[non], k[non]
        src = []
        for x, m, md in ((i, d[0], dn[0]), (j, d[1], dn[1]), (k, d[2], dn[2])):
            src.append(np.where(x < 1, md - 2 + x, np.where(x > m - 2, x - (m - 2), 1 + (x - 1) % (md - 2))))
        bb = np.full_like(i, b)
        st.append(np.stack([bb, i, j, k, np.full_like(i, perm[b]), src[0], src[1], src[2], np.zeros_like(i)], axis=1))
    m = np.ascontiguousarray(np.concatenate(st).astype(np.int32))
    return m, m.copy()


def check_halo_map(dims, entries: np.ndarray, kind: int):
    """Host checks of a halo map, the same the library makes (raises ValueError)."""
    e = np.asarray(entries)
    dims = np.asarray(dims)
    for c0, c1 in ((0, 1), (4, 5)):
        b = e[:, c0]
        if (b < 0).any() or (b >= len(dims)).any():
            raise ValueError("block index")
        for a in range(3):
            x, m = e[:, c1 + a], dims[b, a]
            if (x < -2).any() or (x > m + 1).any():
                raise ValueError("node outside the padded box")

    def interior(b, i, j, k):
        d = dims[b]
        return (i >= 1) & (i <= d[:, 0] - 2) & (j >= 1) & (j <= d[:, 1] - 2) & (k >= 1) & (k <= d[:, 2] - 2)

    if interior(e[:, 0], e[:, 1], e[:, 2], e[:, 3]).any():
        raise ValueError("destination is an interior node")
    if kind == HALO_STAGE:
        out_src = e[:, 8] == 0
        if (~interior(e[out_src, 4], e[out_src, 5], e[out_src, 6], e[out_src, 7])).any():
            raise ValueError("stage-output source is not an interior node")
    key_d = [tuple(r) for r in e[:, 0:4]]
    if len(set(key_d)) != len(key_d):
        raise ValueError("duplicate destination")
    if kind == HALO_WRAP:
        ks = set(key_d)
        if any(tuple(r) in ks for r in e[:, 4:8]):
            raise ValueError("wrap source is also a destination")


# ------------------------------------------------------------------ batch --
class Batch:
    """Many curvilinear blocks of uneven sizes, resident on one GPU and
    advanced together (one persistent stage launch per RK stage)."""

    def __init__(self, dims: Sequence[Tuple[int, int, int]], les: int = 0, inviscid: int = 0, fluxorder: int = 3,
                 eno_order: int = 2, central: int = 2, isothermal: int = 0, s_x: float = 1.0, s_y: float = 1.0,
                 s_z: float = 1.0, ren: float = 3000.0, ma: float = 2.81, pr: float = 0.72, gamma: float = 1.4,
                 dt: float = 0.01, st: float = 1.0, cs_const: float = 0.03, ci: float = 0.06, ratio: float = 0.0,
                 precision: str = "fp64", device: int = 0, calc_sigma: int = 0, visT: int = 0,
                 tref: float = 273.15, twod: int = 0, flux: str = "rusanov", weno_order: int = 3,
                 s_x_min: float = 0.0, s_y_min: float = 0.0, s_z_min: float = 0.0, sigma_thrsh: float = 1e-5,
                 abc: int = 0, max_cs: float = 0.05, i_homo_filter: int = 0, j_homo_filter: int = 0,
                 k_homo_filter: int = 0, testfilter_ik: int = 0, twall: float = 1.0):
        self.lib = _lib.load()
        self.dims = [tuple(int(x) for x in d) for d in dims]
        cfg = CbConfig()
        mx, my, mz = self.dims[0]
        self.lib.cb_config_default(C.byref(cfg), mx, my, mz)
        for k, v in dict(les=les, inviscid=inviscid, fluxorder=fluxorder, eno_order=eno_order, central=central,
                         isothermal=isothermal, s_x=s_x, s_y=s_y, s_z=s_z, ren=ren, ma=ma, pr=pr, gamma=gamma,
                         dt=dt, st=st, cs_const=cs_const, ci=ci, ratio=ratio, device=device,
                         calc_sigma=calc_sigma, visT=visT, tref=tref, twod=twod, weno_order=weno_order,
                         s_x_min=s_x_min, s_y_min=s_y_min, s_z_min=s_z_min, sigma_thrsh=sigma_thrsh,
                         abc=abc, max_cs=max_cs, i_homo_filter=i_homo_filter, j_homo_filter=j_homo_filter,
                         k_homo_filter=k_homo_filter, testfilter_ik=testfilter_ik, twall=twall).items():
            setattr(cfg, k, v)
        cfg.flux = {"rusanov": 0, "roe": 1}[flux] if isinstance(flux, str) else int(flux)
        cfg.precision = {"fp64": _lib.CB_FP64, "mixed": _lib.CB_MIXED}[precision]
        self.cfg = cfg
        flat = (C.c_int * (3 * len(self.dims)))(*[x for d in self.dims for x in d])
        self._b = C.c_void_p()
        rc = self.lib.cb_batch_create(C.byref(cfg), len(self.dims), flat, C.byref(self._b))
        if rc != 0:
            raise ChimeraError(rc, "cb_batch_create failed (see stderr)")

    def _check(self, rc: int):
        if rc != 0:
            msg = self.lib.cb_batch_last_error(self._b)
            raise ChimeraError(rc, msg.decode() if msg else "")

    def shape(self, k: int):
        mx, my, mz = self.dims[k]
        return (mz, my, mx)

    @property
    def interior_nodes(self) -> int:
        return int(self.lib.cb_batch_interior_nodes(self._b))

    @property
    def work_items(self) -> int:
        return int(self.lib.cb_batch_work_items(self._b))

    @property
    def stream(self) -> int:
        return int(self.lib.cb_batch_stream(self._b) or 0)

    def FormMetrics(self, k: int, coor: np.ndarray):
        c = np.ascontiguousarray(coor, dtype=np.float64).reshape(self.shape(k) + (3,))
        self._check(self.lib.cb_batch_set_grid(self._b, k, dptr(c)))

    def set_nvert(self, k: int, nvert: np.ndarray):
        n = np.ascontiguousarray(nvert, dtype=np.float64).reshape(self.shape(k))
        self._check(self.lib.cb_batch_set_nvert(self._b, k, dptr(n)))

    def set_bctype(self, k: int, bctype: Sequence[int]):
        """Face codes of block k (i-lo, i-hi, j-lo, j-hi, k-lo, k-hi), as one
        line of the reference's bcs.dat per block (init.c:556-559): with a
        code other than 7 the block runs its own FormBCS after every stage and
        takes no halo-map destination."""
        bc = (C.c_int * 6)(*[int(x) for x in bctype])
        self._check(self.lib.cb_batch_set_bctype(self._b, k, bc))

    def set_time_index(self, ti: int) -> None:
        """user->ti of the last completed step (the next step runs ti + 1),
        read by the k-lo inflow code 47 (cb_batch_set_time_index)."""
        self._check(self.lib.cb_batch_set_time_index(self._b, int(ti)))

    # ------------------------------------------------------ immersed bodies --
    def set_ibm_surface(self, ibi: int, surface: dict):
        """IBMNodes of body ibi, shared by every block (as Block.set_ibm_surface)."""
        tri = [np.ascontiguousarray(surface[k], dtype=np.int32) for k in ("nv1", "nv2", "nv3")]
        nf = [np.ascontiguousarray(surface[k], dtype=np.float64) for k in ("nf_x", "nf_y", "nf_z")]
        n_v = int(surface["n_v"]) if "n_v" in surface else len(surface["x"])
        self._check(self.lib.cb_batch_ibm_set_surface(self._b, ibi, n_v, len(tri[0]), *[t.ctypes.data for t in tri],
                                                      *[dptr(a) for a in nf]))

    def set_ibm_velocity(self, ibi: int, u: np.ndarray, uold: np.ndarray):
        u = np.ascontiguousarray(u, dtype=np.float64)
        uold = np.ascontiguousarray(uold, dtype=np.float64)
        self._check(self.lib.cb_batch_ibm_set_velocity(self._b, ibi, dptr(u), dptr(uold)))

    def set_ibm_list(self, k: int, ibi: int, info: np.ndarray, coor: np.ndarray):
        """Interpolation list of body ibi on block k (a block with face codes)
        and that block's node coordinates."""
        a = np.ascontiguousarray(info, dtype=_lib.IBM_INFO_DTYPE)
        c = np.ascontiguousarray(coor, dtype=np.float64).reshape(self.shape(k) + (3,))
        self._check(self.lib.cb_batch_ibm_set_list(self._b, k, ibi, a.size, a.ctypes.data if a.size else None,
                                                   dptr(c)))

    def set_ibm_options(self, twoD: int = 0, wallfunction: int = 0):
        self._check(self.lib.cb_batch_ibm_set_options(self._b, twoD, wallfunction))

    def SetInitialCondition(self, k: int, q: np.ndarray):
        a = np.ascontiguousarray(q, dtype=np.float64).reshape(self.shape(k) + (5,))
        self._check(self.lib.cb_batch_upload_state(self._b, k, dptr(a)))

    upload_state = SetInitialCondition

    def Q(self, k: int) -> np.ndarray:
        out = np.empty(self.shape(k) + (5,))
        self._check(self.lib.cb_batch_download_state(self._b, k, dptr(out)))
        return out

    def cfl_dt(self, cfl: float):
        """(dt, lambda_max) for the CFL number `cfl` over every block."""
        dt, lam = C.c_double(), C.c_double()
        self._check(self.lib.cb_batch_cfl_dt(self._b, float(cfl), C.byref(dt), C.byref(lam)))
        return dt.value, lam.value

    def metrics(self, k: int):
        """(csi, eta, zet, aj) of block k as resident on the device."""
        csi, eta, zet = (np.empty(self.shape(k) + (3,)) for _ in range(3))
        aj = np.empty(self.shape(k))
        self._check(self.lib.cb_batch_get_metrics(self._b, k, dptr(csi), dptr(eta), dptr(zet), dptr(aj)))
        return csi, eta, zet, aj

    def set_halo_map(self, kind: int, entries: np.ndarray):
        e = np.ascontiguousarray(entries, dtype=np.int32).reshape(-1, 9)
        self._check(self.lib.cb_batch_set_halo_map(self._b, int(kind), e.shape[0],
                                                   e.ctypes.data_as(C.POINTER(C.c_int))))

    def set_halo_maps(self, maps):
        stage, wrap = maps
        self.set_halo_map(HALO_STAGE, stage)
        self.set_halo_map(HALO_WRAP, wrap)

    def set_exchange(self, kind: int, send: np.ndarray, d_send: int, recv: np.ndarray, d_recv: int):
        """Cross-process exchange lists (see cb_batch_set_exchange): send rows of
        5 (stage) or 4 (wrap) ints, recv rows of 4 ints; d_send / d_recv device
        pointers of caller-owned buffers (5 doubles per entry)."""
        sw = 5 if kind == HALO_STAGE else 4
        s = np.ascontiguousarray(send, dtype=np.int32).reshape(-1, sw)
        r = np.ascontiguousarray(recv, dtype=np.int32).reshape(-1, 4)
        ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))
        self._check(self.lib.cb_batch_set_exchange(self._b, int(kind), s.shape[0], ip(s), C.c_void_p(d_send or None),
                                                   r.shape[0], ip(r), C.c_void_p(d_recv or None)))

    def phase(self, phase: int, stage: int = 0, per_block: bool = False):
        self._check(self.lib.cb_batch_phase(self._b, int(phase), int(stage), 1 if per_block else 0))

    def phase_unpack(self, phase: int):
        self._check(self.lib.cb_batch_phase_unpack(self._b, int(phase)))

    def halo_periodic(self):
        self._check(self.lib.cb_batch_halo_periodic(self._b))

    def RungeKutta(self, nsteps: int = 1, per_block: bool = False, sync: bool = True):
        """nsteps RK steps of every block; per_block: one stage launch per block
        instead of the persistent launch (for comparison)."""
        self._check(self.lib.cb_batch_rk_step(self._b, int(nsteps), 1 if per_block else 0))
        if sync:
            self.sync()

    Flow_Solver = RungeKutta

    def sync(self):
        self._check(self.lib.cb_batch_sync(self._b))

    def autotune(self):
        """(best k-chunk, its stage time in ms)."""
        kc, ms = C.c_int(), C.c_double()
        self._check(self.lib.cb_batch_autotune(self._b, C.byref(kc), C.byref(ms)))
        return kc.value, ms.value

    def close(self):
        if self._b:
            self.lib.cb_batch_destroy(self._b)
            self._b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
