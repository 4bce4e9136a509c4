"""ctypes binding of the C ABI declared in include/qmb_b200.h.

The shared library is loaded from this package directory; if it is missing
the import fails loudly (there is no fallback implementation).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libqmb_b200.so")

QMB_OK = 0
QMB_ERR_INVALID = 1
QMB_ERR_CUDA = 2
QMB_ERR_NOMEM = 3
QMB_ERR_ELL_OVERFLOW = 4
QMB_ERR_NOT_CONVERGED = 5
QMB_ERR_TIMEOUT = 6
QMB_ERR_UNSUPPORTED = 7
QMB_ERR_NO_DEVICE = 8
QMB_ERR_IO = 9
QMB_ERR_CORRUPT = 10

OP_SZ, OP_SP, OP_SM, OP_I = 0, 1, 2, 9
PREC_FP64, PREC_FP32 = 1, 2
MODE_FP64, MODE_MIXED, MODE_FP32 = 0, 1, 2
START_SPLITMIX, START_CURAND = 0, 1
HV_STORED, HV_MATRIX_FREE = 0, 1


class QMBError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"qmb status {status}: {msg}")
        self.status = status


class Geometry(C.Structure):
    _fields_ = [("N1", C.c_int), ("N2", C.c_int), ("n_sub", C.c_int), ("a", C.c_double * 4),
                ("rx", C.POINTER(C.c_double)), ("ry", C.POINTER(C.c_double))]


class SectorDesc(C.Structure):
    _fields_ = [("L", C.c_int), ("n_up", C.c_int), ("n_perm", C.c_int),
                ("perm", C.POINTER(C.c_uint32)), ("spin_flip", C.c_int), ("device", C.c_int)]


class SectorInfo(C.Structure):
    _fields_ = [("n_states", C.c_int64), ("n_orbits", C.c_int64), ("n_active", C.c_int64),
                ("n_ext", C.c_int), ("structured", C.c_int), ("is_real", C.c_int)]


class Terms(C.Structure):
    _fields_ = [("n_terms", C.c_int), ("n_col", C.c_int), ("n_ops", C.POINTER(C.c_int)),
                ("op_code", C.POINTER(C.c_int)), ("op_site", C.POINTER(C.c_int)),
                ("scalar", C.POINTER(C.c_double))]


class HamInfo(C.Structure):
    _fields_ = [("n_rows", C.c_int64), ("nnz_offdiag", C.c_int64), ("padded", C.c_int64),
                ("max_row", C.c_int), ("is_complex", C.c_int), ("n_codes", C.c_int),
                ("coded", C.c_int), ("bytes_fp64", C.c_double), ("bytes_fp32", C.c_double),
                ("coded_fp64", C.c_int)]


class LanczosOpts(C.Structure):
    _fields_ = [("mode", C.c_int), ("max_iter", C.c_int), ("min_iter", C.c_int),
                ("tol", C.c_double), ("reorth", C.c_int), ("start", C.c_int),
                ("seed", C.c_uint64), ("check_every", C.c_int), ("hv", C.c_int),
                ("refine_max_iter", C.c_int), ("want_vector", C.c_int)]


class LanczosResult(C.Structure):
    _fields_ = [("E0", C.c_double), ("E0_low", C.c_double), ("residual", C.c_double),
                ("residual_ref", C.c_double), ("iters", C.c_int), ("iters_low", C.c_int),
                ("n_hv", C.c_int), ("converged", C.c_int), ("ms_total", C.c_double),
                ("ms_hv", C.c_double), ("n_products", C.c_double), ("n_launches", C.c_double)]


class BatchDesc(C.Structure):
    _fields_ = [("n_sectors", C.c_int), ("sectors", C.POINTER(C.c_void_p)),
                ("terms_xy", C.POINTER(Terms)), ("terms_z", C.POINTER(Terms)),
                ("n_sets", C.c_int), ("device", C.c_int)]


class BatchInfo(C.Structure):
    _fields_ = [("rows_total", C.c_int64), ("elems_total", C.c_int64),
                ("bytes_hv_fp64", C.c_double), ("bytes_hv_fp32", C.c_double),
                ("rows_per_block", C.c_int), ("sets_per_thread", C.c_int),
                ("set_stride", C.c_int), ("variant_fp32", C.c_int), ("variant_fp64", C.c_int),
                ("tune_ms_fp32", C.c_float * 8), ("tune_ms_fp64", C.c_float * 8),
                ("ring_slots", C.c_int * 2), ("nnz_total", C.c_int64)]


vp = C.c_void_p
i32 = C.c_int
i64 = C.c_int64
dbl = C.c_double
P = C.POINTER

# name -> (restype, argtypes)
SIGNATURES = {
    "qmb_abi_version": (i32, []),
    "qmb_last_error": (C.c_char_p, []),
    "qmb_status_string": (C.c_char_p, [i32]),
    "qmb_device_count": (i32, []),
    "qmb_l2_gather_probe": (i32, [i64, i32, i64, P(dbl), P(dbl)]),
    "qmb_geometry_sites": (i32, [P(Geometry), vp, vp]),
    "qmb_tstandard_pairs": (i32, [P(Geometry), i32, vp, vp, i32, i32, i32, vp, vp, vp, P(i32)]),
    "qmb_extended_xxx_shells": (i32, [P(Geometry), i32, vp, i32, vp, vp, P(i32)]),
    "qmb_heisenberg_terms": (i32, [P(Geometry), i32, vp, vp, i32, vp, vp, i32, i32, i32, vp, vp,
                                   vp, vp, P(i32)]),
    "qmb_group_elem_arr": (i32, [i32, i32, vp, vp, vp, vp, vp]),
    "qmb_group_translations": (i32, [P(Geometry), vp, vp]),
    "qmb_group_rotations": (i32, [i32, vp, vp, i32, vp, vp, vp]),
    "qmb_terms_from_pairs": (i32, [i32, vp, vp, vp, dbl, dbl, i32, i32, vp, vp, vp, vp, P(i32)]),
    "qmb_sector_create": (i32, [P(SectorDesc), P(vp)]),
    "qmb_sector_destroy": (i32, [vp]),
    "qmb_sector_get_info": (i32, [vp, P(SectorInfo)]),
    "qmb_sector_set_irrep": (i32, [vp, vp, dbl]),
    "qmb_sector_reps": (i32, [vp, vp, i64]),
    "qmb_sector_norms": (i32, [vp, vp, i64]),
    "qmb_sector_active": (i32, [vp, vp, i64]),
    "qmb_sector_orbit_map": (i32, [vp, vp, i64]),
    "qmb_sector_lookup": (i32, [vp, vp, i64, vp, vp]),
    "qmb_ham_create": (i32, [vp, P(Terms), i32, P(vp)]),
    "qmb_ham_destroy": (i32, [vp]),
    "qmb_ham_get_info": (i32, [vp, P(HamInfo)]),
    "qmb_ham_export_ref": (i32, [vp, P(Terms), i32, vp, vp, vp]),
    "qmb_ham_export_nosym": (i32, [i32, i32, P(Terms), i32, vp, vp, vp, i32]),
    "qmb_hv": (i32, [vp, i32, vp, vp, vp]),
    "qmb_hv_host": (i32, [vp, i32, vp, vp]),
    "qmb_hv_matrix_free": (i32, [vp, i32, vp, vp, vp]),
    "qmb_lanczos_default_opts": (None, [P(LanczosOpts)]),
    "qmb_lanczos": (i32, [vp, P(LanczosOpts), P(LanczosResult), vp, i64]),
    "qmb_ground_state": (i32, [vp, vp, i64]),
    "qmb_set_ground_state": (i32, [vp, vp, i64]),
    "qmb_eigvec_from_seed_ref": (i32, [C.c_longlong, vp, vp, i32, i32, i32, vp, vp, vp, i32]),
    "qmb_expval": (i32, [vp, i32, P(Terms), vp, vp]),
    "qmb_sector_save": (i32, [vp, C.c_char_p]),
    "qmb_sector_load": (i32, [C.c_char_p, i32, P(vp)]),
    "qmb_ham_save": (i32, [vp, C.c_char_p]),
    "qmb_ham_load": (i32, [vp, C.c_char_p, P(vp)]),
    "qmb_ref_ell_save": (i32, [C.c_char_p, i64, i32, vp, vp, vp, i32]),
    "qmb_ref_ell_load": (i32, [C.c_char_p, P(i64), P(i32), P(i32), vp, vp, vp, i64]),
    "qmb_lanczos_ref_ell": (i32, [P(C.c_float), i32, i32, i32, C.c_longlong, vp, vp, vp, i32,
                                  vp, i32, P(C.c_float)]),
    "qmb_lanczos_ref_ell_noalloc": (i32, [P(C.c_float), i32, i32, i32, C.c_longlong, vp, vp, vp,
                                          i32, vp, i32, P(C.c_float), vp]),
    "qmb_batch_create": (i32, [P(BatchDesc), P(vp)]),
    "qmb_batch_destroy": (i32, [vp]),
    "qmb_batch_get_info": (i32, [vp, P(BatchInfo)]),
    "qmb_batch_solve": (i32, [vp, vp, vp, P(LanczosOpts), vp, P(LanczosResult)]),
    "qmb_batch_hv": (i32, [vp, i32, vp, vp, vp]),
    "qmb_batch_k1_time": (i32, [vp, i32, i32, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "qmb_batch_layout": (i32, [vp, vp, vp]),
}

_lib = None


def lib():
    """The loaded libqmb_b200.so with signatures applied."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python qmbcuda_b200/build.py` "
                              "(the engine has no fallback implementation)")
        L = C.CDLL(LIB_PATH)
        for name, (rt, at) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = rt
            f.argtypes = at
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != QMB_OK:
        msg = lib().qmb_last_error().decode(errors="replace")
        raise QMBError(status, msg)


def ptr(a: np.ndarray):
    """Host pointer of a C-contiguous numpy array."""
    assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return a.ctypes.data_as(C.c_void_p)


def cplx_buf(a) -> np.ndarray:
    """complex128 array -> contiguous interleaved float64 view."""
    return np.ascontiguousarray(np.asarray(a, dtype=np.complex128)).view(np.float64)


def default_opts(**kw) -> LanczosOpts:
    o = LanczosOpts()
    lib().qmb_lanczos_default_opts(C.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise AttributeError(k)
        setattr(o, k, v)
    return o
