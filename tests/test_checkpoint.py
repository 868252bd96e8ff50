"""Checkpoint files in the reference's PETSc binary layout (main.c:215-304)."""
import numpy as np
import pytest

from chimera_comp_les_b200 import checkpoint as CK


def test_vec_file_layout_and_roundtrip(tmp_path):
    rng = np.random.default_rng(1)
    a = rng.standard_normal((4, 3, 5, 5))
    p = str(tmp_path / "Qfield00007_0.dat")
    CK.write_vec(p, a, 5)
    raw = open(p, "rb").read()
    assert len(raw) == 8 + 8 * a.size
    assert raw[:4] == (1211214).to_bytes(4, "big") and raw[4:8] == a.size.to_bytes(4, "big")
    assert np.frombuffer(raw[8:16], ">f8")[0] == a.reshape(-1)[0]  # natural order, components interleaved
    assert open(p + ".info").read().strip() == "-vecload_block_size 5"
    assert np.array_equal(CK.read_vec(p), a.reshape(-1))


def test_read_rejects_other_files(tmp_path):
    p = tmp_path / "x.dat"
    p.write_bytes(b"\x00\x00\x00\x01\x00\x00\x00\x02")
    with pytest.raises(ValueError):
        CK.read_vec(str(p))


def test_sigma_field_matches_sensor_off_rule():
    s = CK.sigma_field((4, 5, 6), True, 0.3, 0.7, 0.5)
    assert s[0, 0, 0].tolist() == [0.3, 0.7, 0.5]
    assert s[2, 2, 2].tolist() == [0.3, 0.5, 0.5]


@pytest.mark.gpu
def test_block_checkpoint_roundtrip(tmp_path):
    import math

    from chimera_comp_les_b200 import Block
    from chimera_comp_les_b200 import workloads as W
    n = (20, 16, 14)
    coords = W.periodic_grid(n, 2 * math.pi, amp=0.03)
    q = W.tgv_state(coords)
    nv = np.zeros(coords.shape[:3])
    nv[3:6, 4:7, 5:9] = 3.0
    kw = dict(les=1, fluxorder=3, ren=1600.0, ma=0.1, pr=0.71, dt=2e-3)
    with Block(n[0] + 2, n[1] + 2, n[2] + 2, **kw) as a:
        a.FormMetrics(coords)
        a.set_nvert(nv)
        a.SetInitialCondition(q)
        a.RungeKutta(2)
        files = CK.Q_P_Binary_Output(a, 2, 0, str(tmp_path), nvert=nv)
        assert len(files) == 5
        a.RungeKutta(1)
        want = a.Q()
    with Block(n[0] + 2, n[1] + 2, n[2] + 2, **kw) as b:
        b.FormMetrics(coords)
        got_nv = CK.Q_P_Binary_Input(b, 2, 0, str(tmp_path))
        assert np.array_equal(got_nv, nv)
        p = CK.read_vec(files[2]).reshape(b.shape)
        assert np.array_equal(p, b.EqOfState())
        # a restart drops the eddy viscosity of the interrupted step (as the
        # reference's restart does), so the next step differs only through nu_t
        b.RungeKutta(1)
        got = b.Q()
    assert np.isfinite(got).all()
    assert np.max(np.abs(got - want)) < 1e-3 * np.max(np.abs(want))
