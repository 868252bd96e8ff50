"""The CPU baseline leg of the bench (oracle/cpu_baseline.py): the reference's
own RHS + RK stage path, built here against the serial PETSc shim, timed as
P independent processes on k-slabs, with the optimised build and the shipped
-O0 build.  Checked on a small slab: it runs, counts the cell-updates it did,
and names the build it timed."""
import math

import pytest

import oracle as O

pytestmark = pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) not available")

CFG = dict(les=1, inviscid=0, fluxorder=2, s_x=0.0, s_y=0.0, s_z=0.0, ren=1600.0, ma=0.1, pr=0.71, dt=1e-3)


@pytest.mark.parametrize("procs,optimized", [(1, True), (1, False), (2, True)])
def test_reference_slabs_run_and_report(procs, optimized):
    from oracle import cpu_baseline as cb
    r = cb.run(16, steps=1, procs=procs, cfgkw=CFG, optimized=optimized, nz=4)
    assert r["kind"] == "reference"
    assert r["cores"] == procs
    assert r["value"] > 0 and math.isfinite(r["value"])
    # 16 x 16 x 4 interior nodes per process, 2 RK stages (fluxorder 2)
    assert abs(r["value"] * r["seconds"] - procs * 16 * 16 * 4 * 2) < 1e-6 * procs * 16 * 16 * 4 * 2
    assert ("-O3" in r["sample"]) == optimized and ("-O0" in r["sample"]) == (not optimized)
    assert f"{procs} processes" in r["sample"] and "16x16x4" in r["sample"]
