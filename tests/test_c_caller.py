"""The drop-in boundary as a C host sees it: plain C99 programs that include
only include/chimera_b200.h and link libchimera_b200.so.

* The struct layouts the C compiler gives cb_config and cb_ibm_info equal the
  Python ctypes mirror (no GPU needed).
* The call sequence a maintainer adds around RungeKutta (cb_config_default,
  cb_create, cb_set_grid, cb_set_nvert, cb_upload_state, cb_rk_step, cb_sync,
  cb_download_state) compiles and links as C99 and, on a GPU, reproduces the
  oracle's time steps to relative L2 <= 1e-12 per conserved field.
* The reference's multi-block loop through the batched calls (blocks with
  their own face codes beside interface blocks) compiles and links as C99
  and, on a GPU, advances every block exactly as a single-block context with
  the same codes.
"""
import json
import math
import os
import subprocess

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CDIR = os.path.join(REPO, "tests", "c_caller")
INCLUDE = os.path.join(REPO, "include")
CFLAGS = ["-std=c99", "-pedantic", "-Wall", "-Wextra", "-Werror", "-O1", "-I", INCLUDE]


def _lib_dir():
    from chimera_comp_les_b200 import build
    return os.path.dirname(build.build())


def _compile(src, exe, link=False):
    cmd = ["gcc"] + CFLAGS + [os.path.join(CDIR, src), "-o", str(exe)]
    if link:
        d = _lib_dir()
        cmd += ["-L", d, "-lchimera_b200", f"-Wl,-rpath,{d}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_struct_layout_matches_ctypes(tmp_path):
    from chimera_comp_les_b200 import _lib
    exe = _compile("layout.c", tmp_path / "layout")
    lay = json.loads(subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout)
    cfg = lay["cb_config"]
    assert cfg["size"] == __import__("ctypes").sizeof(_lib.CbConfig)
    ct = {name: getattr(_lib.CbConfig, name).offset for name, _ in _lib.CbConfig._fields_}
    assert cfg["fields"] == ct
    info = lay["cb_ibm_info"]
    assert info["size"] == _lib.IBM_INFO_DTYPE.itemsize
    assert info["fields"] == {k: v[1] for k, v in _lib.IBM_INFO_DTYPE.fields.items()}


def test_driver_compiles_and_links_as_c99(tmp_path):
    exe = _compile("rk_driver.c", tmp_path / "rk_driver", link=True)
    assert os.path.exists(exe)


def test_batch_driver_compiles_and_links_as_c99(tmp_path):
    exe = _compile("batch_driver.c", tmp_path / "batch_driver", link=True)
    assert os.path.exists(exe)


@pytest.mark.gpu
def test_c_host_steps_match_oracle(tmp_path):
    import oracle as O
    from chimera_comp_les_b200 import workloads as W
    n = (26, 20, 18)
    coords = W.periodic_grid(n, 2 * math.pi, amp=0.05)
    q0 = W.tgv_state(coords, gamma=1.4, ma=0.1)
    nv = np.zeros(coords.shape[:3])
    opts = dict(les=1, fluxorder=2, s=0.0, ren=1600.0, ma=0.1, pr=0.71, dt=2e-3)
    nsteps = 3
    inp, out = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(inp, "wb") as f:
        np.array([n[0] + 2, n[1] + 2, n[2] + 2], dtype=np.int32).tofile(f)
        for a in (coords, nv, q0):
            np.ascontiguousarray(a, dtype=np.float64).tofile(f)
    exe = _compile("rk_driver.c", tmp_path / "rk_driver", link=True)
    args = [str(exe), str(inp), str(out)] + [str(opts[k]) for k in ("les", "fluxorder", "s", "ren", "ma", "pr", "dt")]
    r = subprocess.run(args + [str(nsteps)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    raw = np.fromfile(out, dtype=np.float64)
    nn = coords.shape[0] * coords.shape[1] * coords.shape[2]
    q_gpu = raw[:5 * nn].reshape(q0.shape)
    p_gpu = raw[5 * nn:].reshape(coords.shape[:3])

    cfg = O.Config(mx=n[0] + 2, my=n[1] + 2, mz=n[2] + 2, les=1, inviscid=0, fluxorder=2, s_x=0.0, s_y=0.0,
                   s_z=0.0, ren=1600.0, ma=0.1, pr=0.71, dt=2e-3)
    ora = O.Oracle(cfg)
    met = ora.metrics(O.to_padded(cfg, coords))
    nvp = ora.fill_ghosts(O.to_padded(cfg, nv))
    st = ora.initial_state(q0)
    ora.steps(nsteps, st, met, nvp)
    q_ref = O.from_padded(st["q"])
    p_ref = O.from_padded(ora.eos(ora.fill_ghosts(st["q"].copy())))[..., 0]
    for fld in range(5):
        assert O.rel_l2(q_gpu[..., fld], q_ref[..., fld]) <= 1e-12, fld
    assert O.rel_l2(p_gpu, p_ref) <= 1e-12


@pytest.mark.gpu
def test_c_host_blocks_match_single_blocks(tmp_path):
    from chimera_comp_les_b200 import Block
    from chimera_comp_les_b200 import workloads as W
    blocks = [((28, 20, 22), (3, 3, 1, 1, 45, 44)), ((22, 18, 20), (7, 7, 1, 1, 7, 7)), ((20, 22, 18), (7,) * 6)]
    opts = dict(les=1, fluxorder=3, s=0.5, ren=500.0, ma=0.3, pr=0.71, dt=2e-3)
    nsteps = 3
    data = []
    for b, (d, bc) in enumerate(blocks):
        coords = W.periodic_grid((d[0] - 2, d[1] - 2, d[2] - 2), 2 * math.pi, amp=0.04)
        data.append((coords, W.random_smooth_state(coords.shape[:3], seed=50 + b, periodic=bc == (7,) * 6)))
    inp, out = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(inp, "wb") as f:
        np.array([len(blocks)], dtype=np.int32).tofile(f)
        for d, bc in blocks:
            np.array(list(d) + list(bc), dtype=np.int32).tofile(f)
        for coords, q in data:
            np.ascontiguousarray(coords, dtype=np.float64).tofile(f)
            np.ascontiguousarray(q, dtype=np.float64).tofile(f)
    exe = _compile("batch_driver.c", tmp_path / "batch_driver", link=True)
    args = [str(exe), str(inp), str(out)] + [str(opts[k]) for k in ("les", "fluxorder", "s", "ren", "ma", "pr", "dt")]
    r = subprocess.run(args + [str(nsteps)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    raw = np.fromfile(out, dtype=np.float64)
    off = 0
    for (d, bc), (coords, q) in zip(blocks, data):
        got = raw[off:off + q.size].reshape(q.shape)
        off += q.size
        with Block(*d, bctype=bc, les=1, fluxorder=3, s_x=0.5, s_y=0.5, s_z=0.5, ren=500.0, ma=0.3, pr=0.71,
                   dt=2e-3) as blk:
            blk.FormMetrics(coords)
            blk.SetInitialCondition(q)
            blk.RungeKutta(nsteps)
            want = blk.Q()
        assert np.array_equal(got, want), bc
    assert off == raw.size
