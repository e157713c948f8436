"""ctypes declarations of include/deco_b200.h.

The library is loaded from this package directory (built in-tree by
deco_b200/build.py).  There is no fallback: if the shared object is missing or
fails to load, the import error says so.
"""
from __future__ import annotations

import ctypes as C
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libdeco_b200.so")

vp = C.c_void_p
ip = C.POINTER(C.c_int)
dp = C.POINTER(C.c_double)


class CprParams(C.Structure):
    _fields_ = [("block_size", C.c_int), ("pressure_id", C.c_int), ("seq", C.c_int), ("weights", C.c_int),
                ("use_drs", C.c_int), ("drs_e_dd", C.c_double), ("drs_e_ps", C.c_double), ("cpd", C.c_int),
                ("tol_zero", C.c_double), ("glo_tol_rel", C.c_double), ("glo_tol_abs", C.c_double),
                ("glo_power", C.c_int), ("loc_tol_rel", C.c_double), ("loc_tol_abs", C.c_double),
                ("loc_power", C.c_int), ("precision", C.c_int), ("glo_type", C.c_int), ("loc_type", C.c_int),
                ("glo_block_size", C.c_int), ("loc_block_size", C.c_int)]


class SolParams(C.Structure):
    _fields_ = [("type", C.c_int), ("reltol", C.c_double), ("restart", C.c_int), ("itmax", C.c_int),
                ("verbosity", C.c_int), ("precision", C.c_int), ("use_x0", C.c_int)]


class SolResult(C.Structure):
    _fields_ = [("iter", C.c_int), ("flag", C.c_int), ("res_abs", C.c_double), ("res_rel", C.c_double),
                ("t_solve_ms", C.c_double), ("restarts", C.c_int), ("t_precond_ms", C.c_double),
                ("t_matvec_ms", C.c_double), ("t_ortho_ms", C.c_double), ("res_rel_orig", C.c_double),
                ("t_dots_ms", C.c_double)]


class BatchResult(C.Structure):
    _fields_ = [("max_iter", C.c_int), ("converged", C.c_int), ("cycles", C.c_int), ("graph", C.c_int),
                ("t_solve_ms", C.c_double)]


# name -> (argtypes, restype); every function in include/deco_b200.h
SIGNATURES = {
    "deco_last_error": ([], C.c_char_p),
    "deco_version": ([], C.c_char_p),
    "deco_launch_count": ([], C.c_longlong),
    "deco_alloc_count": ([], C.c_longlong),
    "deco_ctx_create": ([C.c_int, vp, C.POINTER(vp)], C.c_int),
    "deco_ctx_destroy": ([vp], C.c_int),
    "deco_ctx_sync": ([vp], C.c_int),
    "deco_ctx_stream": ([vp, C.POINTER(vp)], C.c_int),
    "deco_ctx_set_autotune": ([vp, C.c_int], C.c_int),
    "deco_ctx_trim": ([vp], C.c_int),
    "deco_csr_create": ([vp, C.c_int, C.c_int, C.c_int, vp, vp, vp, C.c_int, C.POINTER(vp)], C.c_int),
    "deco_csr_destroy": ([vp], C.c_int),
    "deco_csr_info": ([vp, ip, ip, ip], C.c_int),
    "deco_csr_download": ([vp, vp, vp, vp, vp], C.c_int),
    "deco_csr_set_values": ([vp, vp, vp, C.c_int], C.c_int),
    "deco_csr_make_f32": ([vp, vp], C.c_int),
    "deco_csr_subwarp": ([vp, ip], C.c_int),
    "deco_csr_set_subwarp": ([vp, C.c_int], C.c_int),
    "deco_csr_set_blocks": ([vp, vp, C.c_int], C.c_int),
    "deco_csr_blocks": ([vp, ip, ip], C.c_int),
    "deco_csr_padded": ([vp, ip], C.c_int),
    "deco_csr_product_plan": ([vp, C.c_int, ip, ip], C.c_int),
    "deco_csr_slot_codes": ([vp, ip, ip], C.c_int),
    "deco_spmv": ([vp, vp, vp, vp, C.c_int], C.c_int),
    "deco_spmv_f32": ([vp, vp, vp, vp, C.c_int], C.c_int),
    "deco_residual": ([vp, vp, vp, vp, vp], C.c_int),
    "deco_fsai_create": ([vp, vp, C.c_double, C.c_double, C.c_int, C.c_int, C.POINTER(vp)], C.c_int),
    "deco_fsai_destroy": ([vp], C.c_int),
    "deco_fsai_info": ([vp, ip, ip, ip], C.c_int),
    "deco_fsai_blocks": ([vp, ip, ip, ip], C.c_int),
    "deco_fsai_download": ([vp, vp, vp, vp, vp, vp, vp, vp], C.c_int),
    "deco_fsai_apply": ([vp, vp, vp, vp], C.c_int),
    "deco_fsai_padded": ([vp, ip, ip], C.c_int),
    "deco_fsai_slot_codes": ([vp, ip, ip], C.c_int),
    "deco_fsai_apply_f32": ([vp, vp, vp, vp], C.c_int),
    "deco_fsai_apply_static": ([vp, vp, vp, vp], C.c_int),
    "deco_cpr_create": ([vp, vp, vp, C.POINTER(CprParams), C.POINTER(vp)], C.c_int),
    "deco_cpr_destroy": ([vp], C.c_int),
    "deco_cpr_apply": ([vp, vp, vp, vp], C.c_int),
    "deco_cpr_pressure": ([vp, C.POINTER(vp)], C.c_int),
    "deco_cpr_fsai": ([vp, C.c_int, C.POINTER(vp)], C.c_int),
    "deco_cpr_timings": ([vp, dp], C.c_int),
    "deco_cpr_fixed_diagonals": ([vp, ip], C.c_int),
    "deco_cpr_decouple_rhs": ([vp, vp, vp], C.c_int),
    "deco_gmres_solve": ([vp, vp, vp, vp, vp, C.POINTER(SolParams), C.POINTER(SolResult), vp], C.c_int),
    "deco_csr_transpose": ([vp, vp, C.POINTER(vp)], C.c_int),
    "deco_grad_A_pattern": ([vp, vp, vp, vp, C.c_double, vp], C.c_int),
    "deco_adjoint_create": ([vp, vp, C.POINTER(CprParams), C.POINTER(vp)], C.c_int),
    "deco_adjoint_destroy": ([vp], C.c_int),
    "deco_adjoint_solve": ([vp, vp, vp, vp, C.POINTER(SolParams), C.POINTER(SolResult), vp], C.c_int),
    "deco_adjoint_parts": ([vp, C.POINTER(vp), C.POINTER(vp)], C.c_int),
    "deco_batch_create": ([vp, vp, C.c_int, vp, C.c_int, C.POINTER(CprParams), C.POINTER(vp)], C.c_int),
    "deco_batch_destroy": ([vp], C.c_int),
    "deco_batch_info": ([vp, ip, ip, ip, vp], C.c_int),
    "deco_batch_cpr": ([vp, C.POINTER(vp)], C.c_int),
    "deco_batch_apply": ([vp, vp, vp, vp], C.c_int),
    "deco_batch_solve": ([vp, vp, vp, vp, C.POINTER(SolParams), vp, vp, vp, C.POINTER(BatchResult)], C.c_int),
}

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} not built: run deco_b200.build.build_all() (or __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


class DecoError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"deco error {code}: {msg}")
        self.code = code


def check(rc: int):
    if rc != 0:
        raise DecoError(rc, lib().deco_last_error().decode(errors="replace"))
