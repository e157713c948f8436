"""ctypes binding of oracle/_build/liboracle.so, the plain-C restatement of the
reference's CPR-Krylov path (deco_oracle.c).  TEST INFRASTRUCTURE ONLY."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
_lib = None


class CprParams(C.Structure):
    _fields_ = [("bs", C.c_int), ("p", C.c_int), ("seq", C.c_int), ("weights", C.c_int),
                ("use_drs", C.c_int), ("e_dd", C.c_double), ("e_ps", C.c_double), ("cpd", C.c_int),
                ("tol_zero", C.c_double), ("loc_tol_rel", C.c_double), ("glo_tol_rel", C.c_double),
                ("glo_tol_abs", C.c_double), ("glo_power", C.c_int), ("loc_tol_abs", C.c_double),
                ("loc_power", C.c_int)]


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        vp = C.c_void_p
        L.orc_spmv.argtypes = [C.c_int, vp, vp, vp, vp, vp, C.c_int]
        L.orc_spmv.restype = None
        L.orc_cpr_setup.argtypes = [C.POINTER(CprParams), C.c_int, vp, vp, vp, vp, C.POINTER(vp)]
        L.orc_cpr_apply.argtypes = [vp, vp, vp]
        L.orc_cpr_apply.restype = None
        L.orc_cpr_free.argtypes = [vp]
        L.orc_cpr_free.restype = None
        L.orc_cpr_sizes.argtypes = [vp, vp]
        L.orc_cpr_get.argtypes = [vp, C.c_int, vp, vp, vp, vp, vp, vp]
        L.orc_cpr_get.restype = None
        L.orc_cpr_get_b.argtypes = [vp, vp]
        L.orc_cpr_get_b.restype = None
        L.orc_gmres.argtypes = [vp, C.c_int, C.c_double, C.c_int, C.c_int, vp, C.POINTER(C.c_int),
                                C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int), vp]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data if a is not None else None


_WEIGHTS = {"none": 0, "quasiimpes": 1, "quasiimpes_GE": 2}


def params_from_json(prec: dict) -> CprParams:
    """The `prec` object of a reference parameter file (precond/CPR.hpp:49-65,118,130;
    FSAI keys precond/FSAI/FSAI.hpp:19-20,34)."""
    g, l = prec["prec_glo"], prec["prec_loc"]
    return CprParams(
        bs=int(prec["block_size"]), p=int(prec["pressure_id"]), seq=int(prec["seq"]),
        weights=_WEIGHTS[prec["weights"]], use_drs=int(prec["use_drs"]),
        e_dd=float(prec["drs"]["e_dd"]), e_ps=float(prec["drs"]["e_ps"]), cpd=int(prec["CPD"]),
        tol_zero=float(prec["tol_zero"]), loc_tol_rel=float(l["tol_rel"]),
        glo_tol_rel=float(g["tol_rel"]), glo_tol_abs=float(g["tol_abs"]), glo_power=int(g["power"]),
        loc_tol_abs=float(l["tol_abs"]), loc_power=int(l["power"]))


def spmv(r, c, v, x, bs=1):
    n = len(r) - 1
    y = np.zeros((n + bs - 1) // bs)
    xc = np.ascontiguousarray(x, np.float64)  # kept alive across the call
    lib().orc_spmv(n, _p(r), _p(c), _p(v), _p(xc), _p(y), bs)
    return y


class Cpr:
    def __init__(self, prec: dict, r, c, v, b):
        self.prm = params_from_json(prec)
        self.n = len(r) - 1
        h = C.c_void_p()
        rc = lib().orc_cpr_setup(C.byref(self.prm), self.n, _p(r), _p(c), _p(v), _p(b), C.byref(h))
        if rc != 0:
            raise RuntimeError(f"orc_cpr_setup failed ({rc})")
        self.h = h
        sz = np.zeros(5, np.int64)
        lib().orc_cpr_sizes(self.h, _p(sz))
        self.nnzA, self.np_, self.nnzAp, self.nnzFg, self.nnzFl = (int(t) for t in sz)

    def _get(self, which, n, nz, pair):
        r = np.empty(n + 1, np.int32); c = np.empty(nz, np.int32); v = np.empty(nz)
        if pair:
            r2 = np.empty(n + 1, np.int32); c2 = np.empty(nz, np.int32); v2 = np.empty(nz)
        else:
            r2 = c2 = v2 = None
        lib().orc_cpr_get(self.h, which, _p(r), _p(c), _p(v), _p(r2), _p(c2), _p(v2))
        return ((r, c, v), (r2, c2, v2)) if pair else (r, c, v)

    def decoupled(self):
        r, c, v = self._get(0, self.n, self.nnzA, False)
        b = np.empty(self.n)
        lib().orc_cpr_get_b(self.h, _p(b))
        return r, c, v, b

    def pressure(self):
        return self._get(1, self.np_, self.nnzAp, False)

    def fsai(self, which):
        return self._get(2 if which == 0 else 3, self.n if which == 0 else self.np_,
                         self.nnzFg if which == 0 else self.nnzFl, True)

    def apply(self, rvec):
        x = np.zeros(self.n)
        rc = np.ascontiguousarray(rvec, np.float64)  # kept alive across the call
        lib().orc_cpr_apply(self.h, _p(rc), _p(x))
        return x

    def solve(self, sol: dict):
        left = 1 if sol["type"] == "lgmres" else 0
        itmax = int(sol["itmax"])
        x = np.zeros(self.n)
        resvec = np.zeros(itmax + 1)
        it, fl = C.c_int(), C.c_int()
        ra, rr = C.c_double(), C.c_double()
        lib().orc_gmres(self.h, left, float(sol["reltol"]), int(sol["restart"]), itmax, _p(x), C.byref(it),
                        C.byref(ra), C.byref(rr), C.byref(fl), _p(resvec))
        return dict(x=x, iter=it.value, res_abs=ra.value, res_rel=rr.value, flag=fl.value,
                    resvec=resvec[:it.value])

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_cpr_free(self.h)
            self.h = None
