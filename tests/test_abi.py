"""The C-ABI library loads on a machine without a GPU and exports every
function include/chimera_b200.h declares (no compute calls here)."""
import ctypes
import os
import re

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "chimera_b200.h")


def declared_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(cb_[a-z0-9_]+)\s*\(", txt)))


def _lib_path():
    from chimera_comp_les_b200 import build
    return build.build()


def test_header_declares_core_entry_points():
    names = declared_functions()
    for n in ("cb_create", "cb_destroy", "cb_set_grid", "cb_set_nvert", "cb_upload_state", "cb_rhs",
              "cb_rk_step", "cb_download_state", "cb_eddy_viscosity"):
        assert n in names


def test_library_loads_and_exports_all_declared_symbols():
    lib = ctypes.CDLL(_lib_path())
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    assert lib.cb_abi_version() == 2


def test_config_default_matches_reference_defaults():
    from chimera_comp_les_b200._lib import CbConfig
    lib = ctypes.CDLL(_lib_path())
    c = CbConfig()
    lib.cb_config_default(ctypes.byref(c), 10, 11, 12)
    # init.c:84-92 and main.c:52
    assert (c.mx, c.my, c.mz) == (10, 11, 12)
    assert c.ren == 3000.0 and c.ma == 2.81 and c.gamma == 1.4 and c.pr == 0.72 and c.dt == 0.01
    assert c.central == 2 and c.fluxorder == 3 and c.eno_order == 2
    assert list(c.bctype) == [7] * 6
    assert c.weno_order == 3


def test_product_has_no_cpu_fallback():
    # the product path must not import the oracle
    import chimera_comp_les_b200 as pkg
    src = ""
    for f in os.listdir(os.path.dirname(pkg.__file__)):
        if f.endswith(".py"):
            src += open(os.path.join(os.path.dirname(pkg.__file__), f)).read()
    assert "import oracle" not in src and "from oracle" not in src


def test_every_kernel_is_local_to_the_object_that_compiled_it():
    """The FP64 parity form and the mixed form are compiled with different
    floating-point flags (no FMA contraction / IEEE division versus
    contraction and fast division).  A kernel whose host symbol is global or
    weak can be defined by several objects -- with different flags -- and the
    runtime then launches whichever copy it bound to that symbol.  Every
    kernel symbol of the library must therefore have local binding."""
    import shutil
    import subprocess
    nm = shutil.which("nm")
    if nm is None:
        pytest.skip("nm not available")
    out = subprocess.run([nm, "-C", _lib_path()], capture_output=True, text=True, check=True).stdout
    kern = [ln.split(" ", 2) for ln in out.splitlines() if re.search(r"\bcb::\w+_kernel\b", ln)]
    assert len(kern) > 100, "kernel symbols not found"
    shared = [name for _, kind, name in kern if kind not in ("t", "r", "d", "b")]
    assert not shared, shared[:5]
