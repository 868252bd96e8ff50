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
    p1 = str(tmp_path / "pfield00007_0.dat")
    CK.write_vec(p1, a[..., 0])  # one component: an empty .info side file
    assert open(p1 + ".info").read() == ""


def test_read_rejects_other_files(tmp_path):
    p = tmp_path / "x.dat"
    p.write_bytes(b"\x00\x00\x00\x01\x00\x00\x00\x02")
    with pytest.raises(ValueError):
        CK.read_vec(str(p))


def test_sigma_field_matches_sensor_off_rule():
    s = CK.sigma_field((4, 5, 6), True, 0.3, 0.7, 0.5)
    assert s[0, 0, 0].tolist() == [0.3, 0.7, 0.5]
    assert s[2, 2, 2].tolist() == [0.3, 0.5, 0.5]


# a small LES case with distinct hybrid weights (the interior rule y = z =
# min(s_y, s_z) shows in the Sigma file) and an immersed mask in Nvert
N_CK = (14, 12, 10)
KW_CK = dict(les=1, fluxorder=3, ren=1600.0, ma=0.1, pr=0.71, dt=2e-3, s_x=0.7, s_y=0.4, s_z=0.5)


def _ck_inputs():
    import math

    from chimera_comp_les_b200 import workloads as W
    coords = W.periodic_grid(N_CK, 2 * math.pi, amp=0.03)
    q = W.tgv_state(coords)
    nv = np.zeros(coords.shape[:3])
    nv[3:6, 4:7, 5:9] = 3.0
    return coords, q, nv


def _ref(coords, nv, q=None):
    import oracle as O
    cfg = O.Config(mx=N_CK[0] + 2, my=N_CK[1] + 2, mz=N_CK[2] + 2, **KW_CK)
    ref = O.RefOracle(cfg, coords, io=True)
    ref.set_nvert(nv)
    if q is not None:
        ref.set_state(q)
    return ref


def _files(d):
    return sorted(p.name for p in d.iterdir())


@pytest.mark.skipif(not __import__("oracle").ref_available(), reason="reference build needed")
def test_files_byte_identical_to_reference_writer(tmp_path, monkeypatch):
    """The reference's own Q_P_Binary_Output (main.c:247-304, compiled with
    the shim's binary viewer) and write_fields, given the same vectors,
    write the same files byte for byte: names, order of components, the
    Sigma and Nu_t files of LES, the .info side files."""
    coords, q, nv = _ck_inputs()
    ref = _ref(coords, nv, q)
    ref.steps(2)
    (tmp_path / "ref").mkdir()
    (tmp_path / "py").mkdir()
    monkeypatch.chdir(tmp_path / "ref")
    ref.write_checkpoint(2)
    shape = coords.shape[:3]
    sig = CK.sigma_field(shape, True, KW_CK["s_x"], KW_CK["s_y"], KW_CK["s_z"])
    CK.write_fields(2, 0, str(tmp_path / "py"), ref.Q(), ref.P(), nv, sig, ref.nut())
    names = _files(tmp_path / "ref")
    assert names == _files(tmp_path / "py")
    assert {"Qfield00002_0.dat", "sigma00002_0.dat", "pfield00002_0.dat", "nvfield00002_0.dat",
            "nu_t00002_0.dat"} <= set(names)
    for nm in names:
        assert (tmp_path / "ref" / nm).read_bytes() == (tmp_path / "py" / nm).read_bytes(), nm


@pytest.mark.gpu
@pytest.mark.skipif(not __import__("oracle").ref_available(), reason="reference build needed")
def test_restart_through_either_writer_matches_reference(tmp_path, monkeypatch):
    """Restarts across the two implementations reproduce the reference's own
    post-restart step to relative L2 <= 1e-12 per field: the GPU restarted
    from the reference's files (Q_P_Binary_Input) and the reference restarted
    (RestartApplication, main.c:620-693) from files the GPU path wrote; a
    restart starts from zero eddy viscosity in both, as a fresh process does."""
    from _common import RTOL_L2, per_field_rel_l2
    from chimera_comp_les_b200 import Block
    coords, q, nv = _ck_inputs()
    dims = (N_CK[0] + 2, N_CK[1] + 2, N_CK[2] + 2)
    (tmp_path / "ref").mkdir()
    (tmp_path / "gpu").mkdir()

    # the reference: 2 steps, checkpoint, restart in a fresh set-up, 1 step
    monkeypatch.chdir(tmp_path / "ref")
    ref = _ref(coords, nv, q)
    ref.steps(2)
    ref.write_checkpoint(2)
    ref = _ref(coords, nv)
    ref.restart(2)
    ref.steps(1)
    want = ref.Q()

    # the GPU from the reference's files
    with Block(*dims, **KW_CK) as b:
        b.FormMetrics(coords)
        got_nv = CK.Q_P_Binary_Input(b, 2, 0, str(tmp_path / "ref"))
        assert np.array_equal(got_nv, nv)
        b.RungeKutta(1)
        assert max(per_field_rel_l2(b.Q(), want)) <= RTOL_L2

    # the GPU's own files, read back by the reference
    with Block(*dims, **KW_CK) as a:
        a.FormMetrics(coords)
        a.set_nvert(nv)
        a.SetInitialCondition(q)
        a.RungeKutta(2)
        CK.Q_P_Binary_Output(a, 2, 0, str(tmp_path / "gpu"), nvert=nv)
    monkeypatch.chdir(tmp_path / "gpu")
    ref = _ref(coords, nv)
    ref.restart(2)
    ref.steps(1)
    assert max(per_field_rel_l2(ref.Q(), want)) <= RTOL_L2
