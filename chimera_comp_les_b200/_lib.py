"""ctypes binding of libchimera_b200.so (the C-ABI in include/chimera_b200.h).

The library is loaded from the package directory only.  A missing library is
an error: there is no CPU fallback for the product path.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libchimera_b200.so")

CB_OK, CB_E_ARG, CB_E_CUDA, CB_E_STATE, CB_E_NONFINITE, CB_E_UNSUPPORTED = 0, 1, 2, 3, 4, 5
CB_FP64, CB_MIXED = 0, 1
CB_PHASE_STATE, CB_PHASE_NUT, CB_PHASE_STAGE = 0, 1, 2
CB_IBM_MAX_BODIES = 16

# cb_ibm_info: one entry of an immersed body's interpolation list (the IBMInfo
# fields ibm_interpolation_advanced reads), 144 bytes.
IBM_INFO_DTYPE = np.dtype([
    ("ni", "<i4"), ("nj", "<i4"), ("nk", "<i4"), ("cell", "<i4"),
    ("i1", "<i4"), ("j1", "<i4"), ("k1", "<i4"), ("i2", "<i4"), ("j2", "<i4"), ("k2", "<i4"),
    ("i3", "<i4"), ("j3", "<i4"), ("k3", "<i4"), ("pad", "<i4"),
    ("cr1", "<f8"), ("cr2", "<f8"), ("cr3", "<f8"), ("cs1", "<f8"), ("cs2", "<f8"), ("cs3", "<f8"),
    ("d_s", "<f8"), ("d_i", "<f8"), ("pmin", "<f8", (3,)),
])


class CbConfig(C.Structure):
    _fields_ = [
        ("mx", C.c_int), ("my", C.c_int), ("mz", C.c_int), ("bctype", C.c_int * 6),
        ("les", C.c_int), ("inviscid", C.c_int), ("fluxorder", C.c_int), ("eno_order", C.c_int),
        ("central", C.c_int), ("isothermal", C.c_int),
        ("s_x", C.c_double), ("s_y", C.c_double), ("s_z", C.c_double),
        ("ren", C.c_double), ("ma", C.c_double), ("pr", C.c_double), ("gamma", C.c_double),
        ("dt", C.c_double), ("st", C.c_double), ("cs_const", C.c_double), ("ci", C.c_double),
        ("ratio", C.c_double), ("precision", C.c_int), ("device", C.c_int),
        ("calc_sigma", C.c_int), ("s_x_min", C.c_double), ("s_y_min", C.c_double), ("s_z_min", C.c_double),
        ("sigma_thrsh", C.c_double), ("flux", C.c_int), ("max_cs", C.c_double), ("twall", C.c_double),
        ("twod", C.c_int), ("i_homo_filter", C.c_int), ("j_homo_filter", C.c_int), ("k_homo_filter", C.c_int),
        ("testfilter_ik", C.c_int), ("visT", C.c_int), ("tref", C.c_double), ("abc", C.c_int),
        ("weno_order", C.c_int),
    ]


_lib = None


class ChimeraError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"chimera_b200 error {code}: {msg}")
        self.code = code


def load(path: str = LIB_PATH) -> C.CDLL:
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(
            f"{path} is missing: build it with `python -m chimera_comp_les_b200.build` "
            "(nvcc, sm_100a); the product has no CPU fallback")
    lib = C.CDLL(path)
    P = C.c_void_p
    D = C.POINTER(C.c_double)
    lib.cb_abi_version.restype = C.c_int
    lib.cb_config_default.argtypes = [C.POINTER(CbConfig), C.c_int, C.c_int, C.c_int]
    lib.cb_create.argtypes = [C.POINTER(CbConfig), C.POINTER(P)]
    lib.cb_destroy.argtypes = [P]
    lib.cb_destroy.restype = None
    for name, args in [
        ("cb_set_grid", [P, D]), ("cb_set_metrics", [P, D, D, D, D]), ("cb_get_metrics", [P, D, D, D, D]), ("cb_set_nvert", [P, D]),
        ("cb_upload_state", [P, D]), ("cb_download_state", [P, D, D]), ("cb_rhs", [P, C.c_int, D]),
        ("cb_calc_ucat", [P]), ("cb_eddy_viscosity", [P]), ("cb_get_nut", [P, D]), ("cb_get_cs", [P, D]),
        ("cb_rk_step", [P, C.c_int]), ("cb_sync", [P]), ("cb_capture_graph", [P]),
        ("cb_timing_enable", [P, C.c_int]),
        ("cb_timing_read", [P, D, C.POINTER(C.c_int), D, C.POINTER(C.c_int)]),
    ]:
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = C.c_int
    lib.cb_autotune.argtypes = [P, C.c_int, C.POINTER(C.c_int), D, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    lib.cb_autotune.restype = C.c_int
    lib.cb_cfl_dt.argtypes = [P, C.c_double, D, D]
    lib.cb_cfl_dt.restype = C.c_int
    lib.cb_rhs_noalloc.argtypes = [C.POINTER(CbConfig), P, P, P, P, P, P]
    lib.cb_rhs_noalloc.restype = C.c_int
    lib.cb_stream.argtypes = [P]
    lib.cb_stream.restype = P
    lib.cb_interior_nodes.argtypes = [P]
    lib.cb_interior_nodes.restype = C.c_longlong
    lib.cb_stages.argtypes = [P]
    lib.cb_stages.restype = C.c_int
    lib.cb_launches_per_step.argtypes = [P]
    lib.cb_launches_per_step.restype = C.c_int
    lib.cb_last_error.argtypes = [P]
    lib.cb_last_error.restype = C.c_char_p
    for name, args in [("cb_upload_state_async", [P, P]), ("cb_download_state_async", [P, P]),
                       ("cb_join_transfers", [P])]:
        getattr(lib, name).argtypes = args
        getattr(lib, name).restype = C.c_int
    lib.cb_set_time_index.argtypes = [P, C.c_int]
    lib.cb_set_time_index.restype = C.c_int
    lib.cb_pipe_peaks.argtypes = [C.c_int, D, D]
    lib.cb_pipe_peaks.restype = C.c_int
    # immersed bodies
    for name, args in [
        ("cb_ibm_set_surface", [P, C.c_int, C.c_int, C.c_int, P, P, P, D, D, D]),
        ("cb_ibm_set_velocity", [P, C.c_int, D, D]), ("cb_ibm_set_list", [P, C.c_int, C.c_int, P, D]),
        ("cb_ibm_count", [P, C.c_int]), ("cb_ibm_set_options", [P, C.c_int, C.c_int]),
        ("cb_ibm_interpolate", [P, C.c_int, C.c_int]), ("cb_ibm_get_ustar", [P, C.c_int, D]),
    ]:
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = C.c_int
    # batched multi-block form
    I = C.c_int
    IP = C.POINTER(C.c_int)
    lib.cb_batch_create.argtypes = [C.POINTER(CbConfig), I, IP, C.POINTER(P)]
    lib.cb_batch_create.restype = I
    lib.cb_batch_destroy.argtypes = [P]
    lib.cb_batch_destroy.restype = None
    lib.cb_batch_last_error.argtypes = [P]
    lib.cb_batch_last_error.restype = C.c_char_p
    lib.cb_batch_interior_nodes.argtypes = [P]
    lib.cb_batch_interior_nodes.restype = C.c_longlong
    lib.cb_batch_stream.argtypes = [P]
    lib.cb_batch_stream.restype = P
    lib.cb_batch_work_items.argtypes = [P]
    lib.cb_batch_work_items.restype = I
    for name, args in [
        ("cb_batch_set_grid", [P, I, D]), ("cb_batch_set_nvert", [P, I, D]),
        ("cb_batch_set_bctype", [P, I, IP]), ("cb_batch_set_time_index", [P, I]),
        ("cb_batch_ibm_set_surface", [P, I, I, I, P, P, P, D, D, D]),
        ("cb_batch_ibm_set_velocity", [P, I, D, D]), ("cb_batch_ibm_set_list", [P, I, I, I, P, D]),
        ("cb_batch_ibm_set_options", [P, I, I]),
        ("cb_batch_upload_state", [P, I, D]), ("cb_batch_download_state", [P, I, D]),
        ("cb_batch_get_metrics", [P, I, D, D, D, D]),
        ("cb_batch_set_halo_map", [P, I, C.c_longlong, IP]), ("cb_batch_halo_periodic", [P]),
        ("cb_batch_rk_step", [P, I, I]), ("cb_batch_sync", [P]), ("cb_batch_autotune", [P, IP, D]),
        ("cb_batch_set_exchange", [P, I, C.c_longlong, IP, P, C.c_longlong, IP, P]),
        ("cb_batch_phase", [P, I, I, I]), ("cb_batch_phase_unpack", [P, I]),
        ("cb_batch_cfl_dt", [P, C.c_double, D, D]),
    ]:
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = I
    _lib = lib
    return lib


def dptr(a):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(C.c_double))
