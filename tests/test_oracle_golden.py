"""The oracle restatement reproduces the reference's own outputs (golden
fixtures generated by running rhs.c/les.c/metrics.c/solvers.c via the PETSc
shim)."""
import numpy as np
import pytest

from _common import RTOL_L2, golden_names, load_golden, oracle_run, per_field_rel_l2

NAMES = golden_names()


def test_fixtures_present():
    assert len(NAMES) >= 5


@pytest.mark.parametrize("name", NAMES)
def test_oracle_matches_reference_golden(name):
    cfg, meta, g = load_golden(name)
    out = oracle_run(cfg, g["coords"], g["q"], g["nvert"], steps=meta["steps"])
    for k in ("csi", "eta", "zet", "aj"):
        ref = g["metrics_" + k]
        got = out["metrics"][k]
        assert np.array_equal(got.reshape(ref.shape), ref), k
    if "nut" in g:
        assert np.max(np.abs(out["nut"] - g["nut"])) <= 1e-15 * max(1.0, np.abs(g["nut"]).max())
    assert max(per_field_rel_l2(out["rhs"], g["rhs"])) <= 1e-14
    assert max(per_field_rel_l2(out["q_steps"], g["q_steps"])) <= 1e-14
