"""Loader of libsifelgpu.so (the sm_100a CUDA library, built in-tree).

There is no CPU fallback: if the library cannot be built or loaded, or no
CUDA device is present when a solve runs, the call raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsifelgpu.so")

_lib = None

OK, NOT_CONVERGED, BREAKDOWN, BAD_INPUT, CUDA_ERROR, ZERO_RHS = range(6)
STATUS_NAMES = {0: "OK", 1: "NOT_CONVERGED", 2: "BREAKDOWN", 3: "BAD_INPUT", 4: "CUDA_ERROR", 5: "ZERO_RHS"}
CRIT_SCR_PREC, CRIT_CR_PREC, CRIT_TRUE = 0, 1, 2
FP64, MIXED = 0, 1
PREC_NONE, PREC_JACOBI, PREC_AGG = 0, 1, 101
NOALLOC_MAX_N = 131072  # SGPU_NOALLOC_MAX_N of include/sifelgpu.h


class SolveInfo(C.Structure):
    _fields_ = [
        ("iterations", C.c_int64),
        ("refinements", C.c_int64),
        ("crit_value", C.c_double),
        ("rh_over_ff", C.c_double),
        ("true_relres", C.c_double),
        ("setup_ms", C.c_double),
        ("solve_ms", C.c_double),
        ("spmv_bytes", C.c_double),
        ("spmv_format", C.c_int32),
        ("spmv_variant", C.c_int32),
        ("fallback", C.c_int32),
        ("tile_rows", C.c_int32),
        ("precond_setup_ms", C.c_double),
        ("precond_levels", C.c_int32),
        ("precond_coarse_n", C.c_int32),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Mesh(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("ndofn", C.c_int32),
        ("nn", C.c_int64),
        ("coords", C.c_void_p),
        ("ne", C.c_int64),
        ("elems", C.c_void_p),
        ("cn", C.c_void_p),
        ("emat", C.c_void_p),
        ("thick", C.c_void_p),
        ("rho", C.c_void_p),
        ("dmat", C.c_void_p),
    ]


class AssemblyInfo(C.Structure):
    _fields_ = [
        ("n", C.c_int64),
        ("negm_scr", C.c_int64),
        ("nnz_full", C.c_int64),
        ("colours", C.c_int32),
        ("pattern_ms", C.c_double),
        ("integrate_ms", C.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


ELEM_HEX8, ELEM_QUAD4, ELEM_HEX8T_K, ELEM_HEX8T_C, ELEM_TET4, ELEM_TRI3, ELEM_HEX20, ELEM_QUAD8 = range(8)


class DeckView(C.Structure):
    _fields_ = [
        ("kind", C.c_int32), ("ndofn", C.c_int32), ("nne", C.c_int32), ("mtype", C.c_int32),
        ("nn", C.c_int64), ("ne", C.c_int64), ("n", C.c_int64),
        ("nmat", C.c_int32), ("nmatp", C.c_int32), ("nlc", C.c_int32), ("storage", C.c_int32),
        ("precond", C.c_int32), ("iv", C.c_int32), ("ni", C.c_int64), ("res", C.c_double),
        ("parse_ms", C.c_double),
        ("coords", C.c_void_p), ("elems", C.c_void_p), ("dofflag", C.c_void_p), ("cn", C.c_void_p),
        ("emat_id", C.c_void_p), ("mats", C.c_void_p), ("thick", C.c_void_p), ("loads", C.c_void_p),
        ("problem", C.c_int32), ("tform", C.c_int32), ("alpha", C.c_double), ("t0", C.c_double),
        ("t1", C.c_double), ("dt", C.c_double), ("rnode", C.c_void_p), ("rho", C.c_void_p),
    ]


class SgpuError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


_P = np.ctypeslib.ndpointer
_pL = _P(np.int64, flags="C_CONTIGUOUS")
_pD = _P(np.float64, flags="C_CONTIGUOUS")
_i64, _i32, _dbl, _vp = C.c_int64, C.c_int32, C.c_double, C.c_void_p

# every symbol the public header declares, with its ctypes signature
SIGNATURES = {
    "sgpu_scr_cg_prec": ([_i64, _pL, _pL, _pD, _pD, _pD, _i64, _dbl, C.POINTER(_i64), C.POINTER(_dbl), _dbl,
                          _i64, _i32, C.POINTER(SolveInfo)], C.c_int),
    "sgpu_cr_cg_prec": ([_i64, _pL, _pL, _pD, _pD, _pD, _i64, _dbl, C.POINTER(_i64), C.POINTER(_dbl), _dbl,
                         _i64, _i32, _i32, C.POINTER(SolveInfo)], C.c_int),
    "sgpu_matrix_create": ([_i64, _pL, _pL, _pD, _i32, C.POINTER(_vp)], C.c_int),
    "sgpu_matrix_update_values": ([_vp, _pD], C.c_int),
    "sgpu_matrix_destroy": ([_vp], C.c_int),
    "sgpu_matrix_info": ([_vp, C.POINTER(_i64), C.POINTER(_i64)], C.c_int),
    "sgpu_matrix_download": ([_vp, _i32, _vp, _vp, _vp, C.POINTER(_i64)], C.c_int),
    "sgpu_matrix_mxv": ([_vp, _pD, _pD], C.c_int),
    "sgpu_matrix_mxv_d": ([_vp, _vp, _vp], C.c_int),
    "sgpu_matrix_pcg": ([_vp, _pD, _pD, _i64, _dbl, _dbl, _i64, _i32, _i32, _i32, C.POINTER(_i64),
                         C.POINTER(_dbl), C.POINTER(SolveInfo)], C.c_int),
    "sgpu_matrix_pcg_d": ([_vp, _vp, _vp, _i64, _dbl, _dbl, _i64, _i32, _i32, _i32, C.POINTER(_i64),
                           C.POINTER(_dbl), C.POINTER(SolveInfo)], C.c_int),
    "sgpu_matrix_set_stream": ([_vp, _vp], C.c_int),
    "sgpu_matrix_mxv32_d": ([_vp, _vp, _vp], C.c_int),
    "sgpu_matrix_spmv_plan": ([_vp, _i32, C.POINTER(_dbl), C.POINTER(_i32), C.POINTER(_i32)], C.c_int),
    "sgpu_matrix_set_spmv": ([_vp, _i32, _i32, _i32], C.c_int),
    "sgpu_matrix_set_nullspace": ([_vp, _i32, _pD], C.c_int),
    "sgpu_matrix_precond_clear": ([_vp], C.c_int),
    "sgpu_matrix_set_rigid_body_modes": ([_vp, _i64, _i32, _vp, _vp], C.c_int),
    "sgpu_csr_pcg_noalloc_d": ([_i32, _vp, _vp, _vp, _vp, _vp, _i64, _dbl, _dbl, _i64, _vp, C.POINTER(_i64),
                                C.POINTER(_dbl), C.POINTER(_i64)], C.c_int),
    "sgpu_assembly_lift": ([_vp, _pD, _pD], C.c_int),
    "sgpu_matrix_combine": ([_vp, _vp, _dbl, _dbl, C.POINTER(_vp)], C.c_int),
    "sgpu_transient_dform": ([_vp, _vp, _pD, _pD, _pD, _dbl, _dbl, _i64, _i64, _dbl, _dbl, _i64, _i32, _i32, _vp,
                              C.POINTER(SolveInfo)], C.c_int),
    "sgpu_transient_vform": ([_vp, _vp, _pD, _pD, _pD, _dbl, _dbl, _i64, _i64, _dbl, _dbl, _i64, _i32, _i32, _vp,
                              C.POINTER(SolveInfo)], C.c_int),
    "sgpu_matrix_pcg_multi": ([_vp, _i32, _pD, _pD, _i64, _dbl, _dbl, _i64, _vp, _vp, _vp, C.POINTER(SolveInfo)],
                              C.c_int),
    "sgpu_matrix_pcg_multi_agg": ([_vp, _i32, _pD, _pD, _i64, _dbl, _dbl, _i64, _i32, _vp, _vp, _vp,
                                   C.POINTER(SolveInfo)], C.c_int),
    "sgpu_matrix_pcg_batch_agg": ([_vp, _i32, _pL, _pD, _pD, _i64, _dbl, _dbl, _i32, _vp, _vp, _vp, _vp,
                                   C.POINTER(SolveInfo)], C.c_int),
    "sgpu_matrix_pcg_batch": ([_vp, _i32, _pL, _pD, _pD, _i64, _dbl, _dbl, _i32, _vp, _vp, _vp, _vp,
                               C.POINTER(SolveInfo)], C.c_int),
    "sgpu_assemble": ([C.POINTER(Mesh), C.POINTER(_vp), C.POINTER(AssemblyInfo)], C.c_int),
    "sgpu_reassemble": ([_vp, _i32, _vp, _vp, C.POINTER(AssemblyInfo)], C.c_int),
    "sgpu_assemble_copy": ([_vp, _i32, _vp, _vp, C.POINTER(_vp), C.POINTER(AssemblyInfo)], C.c_int),
    "sgpu_deck_read_mefel": ([C.c_char_p, _i32, C.POINTER(_vp)], C.c_int),
    "sgpu_deck_read_trfel": ([C.c_char_p, _i32, C.POINTER(_vp)], C.c_int),
    "sgpu_deck_get": ([_vp, C.POINTER(DeckView)], C.c_int),
    "sgpu_deck_mesh": ([_vp, C.POINTER(Mesh)], C.c_int),
    "sgpu_deck_rhs": ([_vp, _i32, _pD], C.c_int),
    "sgpu_deck_prescribed": ([_vp, _i32, _pD, C.POINTER(_i64)], C.c_int),
    "sgpu_mesh_element_loads": ([C.POINTER(Mesh), _i64, _vp, _vp, _vp, _pD], C.c_int),
    "sgpu_deck_free": ([_vp], None),
    "sgpu_last_error": ([], C.c_char_p),
    "sgpu_version": ([], C.c_char_p),
    "sgpu_kernel_launches": ([], C.c_int64),
}


def lib():
    """Load (building first if absent) libsifelgpu.so."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            from . import build as _b
            _b.build()
        L = C.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def last_error() -> str:
    return lib().sgpu_last_error().decode()


def check(status, allowed=(OK,)):
    if status not in allowed:
        raise SgpuError(status, last_error())
    return status


def kernel_launches() -> int:
    return int(lib().sgpu_kernel_launches())
