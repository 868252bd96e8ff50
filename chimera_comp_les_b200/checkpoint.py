"""Checkpoint files in the reference's layout: PETSc binary vectors as written
by ``Q_P_Binary_Output`` and read by ``Q_P_Binary_Input`` (main.c:215-304).

File names: ``Qfield%05d_%1d.dat`` (5 per node), ``pfield%05d_%1d.dat``,
``nvfield%05d_%1d.dat``, and with LES ``nu_t%05d_%1d.dat`` and
``sigma%05d_%1d.dat`` (3 per node), with the time step and the block number.
Each is one PETSc binary Vec: big-endian int32 class id 1211214
(VEC_FILE_CLASSID), int32 global length, then the values as big-endian
float64 in the DMDA's natural order (i fastest, components interleaved) --
the layout PETSc's VecView writes for a DMDA vector on a binary viewer.  The
viewer also opens a ``.info`` side file with every file it writes, to which
VecView adds ``-vecload_block_size <n>`` for an n-component vector (empty for
one component).  The PETSc library is not vendored with the reference; this
is its documented binary format (PETSc 3.12, main.c:4).
"""
from __future__ import annotations

import os
from typing import Optional

import numpy as np

VEC_FILE_CLASSID = 1211214


def write_vec(path: str, a: np.ndarray, block_size: int = 1) -> None:
    """One PETSc binary Vec (natural order, interleaved components)."""
    flat = np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
    with open(path, "wb") as f:
        f.write(np.array([VEC_FILE_CLASSID, flat.size], dtype=">i4").tobytes())
        f.write(flat.astype(">f8").tobytes())
    with open(path + ".info", "w") as f:
        if block_size > 1:
            f.write(f"-vecload_block_size {block_size}\n")


def read_vec(path: str) -> np.ndarray:
    """Values of a PETSc binary Vec file (float64, natural order)."""
    with open(path, "rb") as f:
        head = np.frombuffer(f.read(8), dtype=">i4")
        if head.size != 2 or int(head[0]) != VEC_FILE_CLASSID:
            raise ValueError(f"{path}: not a PETSc binary Vec (class id {head[:1]})")
        n = int(head[1])
        data = np.frombuffer(f.read(8 * n), dtype=">f8")
        if data.size != n:
            raise ValueError(f"{path}: truncated ({data.size} of {n} values)")
    return data.astype(np.float64)


def _name(stem: str, ti: int, block: int, directory: str) -> str:
    return os.path.join(directory, "%s%5.5d_%1.1d.dat" % (stem, ti, block))


def sigma_field(shape, les: bool, s_x: float, s_y: float, s_z: float) -> np.ndarray:
    """The reference's Sigma vector with the sensor off (rhs.c:3330-3332 and the
    post-step 3421-3433): (s_x, s_y, s_z) on every node, then on interior nodes
    y = z = min(s_y, s_z)."""
    mz, my, mx = shape
    sig = np.empty(shape + (3,))
    sig[..., 0], sig[..., 1], sig[..., 2] = s_x, s_y, s_z
    m = min(s_y, s_z)
    sig[1:-1, 1:-1, 1:-1, 1] = m
    sig[1:-1, 1:-1, 1:-1, 2] = m
    return sig


def write_fields(ti: int, this: int, directory: str, q: np.ndarray, p: np.ndarray, nvert: np.ndarray,
                 sigma: Optional[np.ndarray] = None, nut: Optional[np.ndarray] = None):
    """The files of main.c:247-304 from natural-order arrays, in its order:
    Qfield, sigma (LES), pfield, nvfield, nu_t (LES); the averaging files of
    -averaging are not written.  Returns the paths."""
    out = []
    for stem, a, bs in (("Qfield", q, 5), ("sigma", sigma, 3), ("pfield", p, 1), ("nvfield", nvert, 1),
                        ("nu_t", nut, 1)):
        if a is None:
            continue
        path = _name(stem, ti, this, directory)
        write_vec(path, a, bs)
        out.append(path)
    return out


def Q_P_Binary_Output(block, ti: int, this: int = 0, directory: str = ".", nvert: Optional[np.ndarray] = None):
    """Writes the checkpoint of a ``solver.Block`` (Q, P from the EOS, nvert,
    and with LES nu_t and Sigma) as main.c:247-304 does; returns the paths."""
    q = np.empty(block.shape + (5,))
    p = np.empty(block.shape)
    block.download(q, p)
    nv = np.zeros(block.shape) if nvert is None else np.asarray(nvert, dtype=np.float64).reshape(block.shape)
    cfg = block.cfg
    les = bool(cfg.les)
    sig = sigma_field(block.shape, True, cfg.s_x, cfg.s_y, cfg.s_z) if les else None
    return write_fields(ti, this, directory, q, p, nv, sig, block.nu_t() if les else None)


def Q_P_Binary_Input(block, ti: int, this: int = 0, directory: str = ".") -> np.ndarray:
    """Reads Qfield / nvfield of step ti (main.c:215-245) into the block
    (nvert first, then Q, which also resets Qold and the eddy viscosity as
    the reference's restart does); returns the nvert array."""
    n = int(np.prod(block.shape))
    nv = read_vec(_name("nvfield", ti, this, directory))
    q = read_vec(_name("Qfield", ti, this, directory))
    if nv.size != n or q.size != 5 * n:
        raise ValueError("checkpoint size does not match the block")
    nv = nv.reshape(block.shape)
    block.set_nvert(nv)
    block.SetInitialCondition(q.reshape(block.shape + (5,)))
    return nv
