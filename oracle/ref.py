"""ctypes binding of oracle/_ref/libdeco_ref.so: the reference's own CPR / FSAI /
SOL code compiled from its sources by oracle/ref/Makefile.

TEST INFRASTRUCTURE ONLY — used by tests/, __graft_entry__.smoke() and the CPU
baseline legs of bench.py as the checker; never by the product.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libdeco_ref.so")
# where the reference's sources are (a checkout of amavliut/deco); without it the
# prebuilt oracle/_ref library is used as it is
REF_SRC = os.environ.get("DECO_REFERENCE", "")

_lib = None


def openblas_dir() -> str:
    """Directory of the OpenBLAS shared object that provides LAPACKE: DECO_OPENBLAS_DIR,
    else the opencv wheel's bundled copy in this Python's site-packages."""
    d = os.environ.get("DECO_OPENBLAS_DIR", "")
    if d:
        return d
    import glob
    import sysconfig
    for base in {sysconfig.get_paths()["purelib"], sysconfig.get_paths()["platlib"]}:
        hits = sorted(glob.glob(os.path.join(base, "opencv_python_headless.libs", "libopenblas*.so")))
        if hits:
            return os.path.dirname(hits[0])
    raise RuntimeError("no OpenBLAS shared object found: set DECO_OPENBLAS_DIR to the directory of libopenblas*.so")


def build(quiet=True, src: str | None = None) -> bool:
    """Compile the reference into oracle/_ref from its sources at `src` (default
    DECO_REFERENCE); without sources, report whether a prebuilt library exists."""
    src = src or REF_SRC
    if not src or not os.path.isdir(src):
        return os.path.exists(LIB)
    subprocess.run(["make", "-s" if quiet else "-k", "-C", os.path.join(HERE, "ref"), f"REF={src}",
                    f"OBLASDIR={openblas_dir()}"], check=True)
    return os.path.exists(LIB)


def available() -> bool:
    return os.path.exists(LIB)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        # OpenBLAS (pthreads build) must not start its own threads inside the
        # reference's OpenMP loops (FSAI local solves call LAPACKE per row):
        # single-threaded BLAS, and no per-call "OpenMP loop" warning
        os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
        L = C.CDLL(LIB)
        vp, ip, dp = C.c_void_p, C.c_void_p, C.c_void_p
        L.ref_spmv.argtypes = [C.c_int, ip, ip, dp, dp, dp, C.c_int]
        L.ref_spmv.restype = None
        L.ref_filter.argtypes = [C.c_int, ip, ip, dp, C.c_double, C.c_int, C.POINTER(C.c_int), ip, ip, dp]
        L.ref_filter.restype = None
        L.ref_fsai_create.argtypes = [C.c_int, ip, ip, dp, C.c_double, C.c_double, C.c_int]
        L.ref_fsai_create.restype = vp
        L.ref_fsai_nnz.argtypes = [vp]
        L.ref_fsai_setup_time.argtypes = [vp]
        L.ref_fsai_setup_time.restype = C.c_double
        L.ref_fsai_get.argtypes = [vp, ip, ip, dp, ip, ip, dp]
        L.ref_fsai_get.restype = None
        L.ref_fsai_apply.argtypes = [vp, dp, dp]
        L.ref_fsai_apply.restype = None
        L.ref_fsai_destroy.argtypes = [vp]
        L.ref_fsai_destroy.restype = None
        L.ref_cpr_create.argtypes = [C.c_char_p, C.c_int, ip, ip, dp, dp]
        L.ref_cpr_create.restype = vp
        L.ref_cpr_setup_time.argtypes = [vp]
        L.ref_cpr_setup_time.restype = C.c_double
        L.ref_cpr_sizes.argtypes = [vp, C.c_void_p]
        L.ref_cpr_sizes.restype = None
        L.ref_cpr_get_A.argtypes = [vp, ip, ip, dp, dp]
        L.ref_cpr_get_A.restype = None
        L.ref_cpr_get_Ap.argtypes = [vp, ip, ip, dp]
        L.ref_cpr_get_Ap.restype = None
        L.ref_cpr_get_fsai.argtypes = [vp, C.c_int, ip, ip, dp, ip, ip, dp]
        L.ref_cpr_apply.argtypes = [vp, dp, dp]
        L.ref_cpr_apply.restype = None
        L.ref_solve.argtypes = [vp, C.c_char_p, dp, C.POINTER(C.c_int), C.POINTER(C.c_double),
                                C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(C.c_double)]
        L.ref_cpr_destroy.argtypes = [vp]
        L.ref_cpr_destroy.restype = None
        L.ref_num_threads.restype = C.c_int
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data if a is not None else None


def spmv(r, c, v, x, bs=1):
    n = len(r) - 1
    y = np.zeros((n + bs - 1) // bs, np.float64)
    xc = np.ascontiguousarray(x, np.float64)  # kept alive across the call
    lib().ref_spmv(n, _p(r), _p(c), _p(v), _p(xc), _p(y), bs)
    return y


def filter(r, c, v, tol, relative):
    n = len(r) - 1
    nz = C.c_int()
    ro = np.empty(n + 1, np.int32)
    co = np.empty(len(c), np.int32)
    vo = np.empty(len(v), np.float64)
    lib().ref_filter(n, _p(r), _p(c), _p(v), tol, int(relative), C.byref(nz), _p(ro), _p(co), _p(vo))
    return ro, co[:nz.value].copy(), vo[:nz.value].copy()


class Fsai:
    """FSAI(const ptree&, shared_ptr<CSR>) of precond/FSAI/FSAI.hpp:14-37."""

    def __init__(self, r, c, v, tol_rel=0.0, tol_abs=0.0, power=1):
        self.n = len(r) - 1
        self.h = lib().ref_fsai_create(self.n, _p(r), _p(c), _p(v), tol_rel, tol_abs, power)
        self.setup_time = lib().ref_fsai_setup_time(self.h)

    def factors(self):
        nz = lib().ref_fsai_nnz(self.h)
        n = self.n
        Lr, Ur = np.empty(n + 1, np.int32), np.empty(n + 1, np.int32)
        Lc, Uc = np.empty(nz, np.int32), np.empty(nz, np.int32)
        Lv, Uv = np.empty(nz), np.empty(nz)
        lib().ref_fsai_get(self.h, _p(Lr), _p(Lc), _p(Lv), _p(Ur), _p(Uc), _p(Uv))
        return (Lr, Lc, Lv), (Ur, Uc, Uv)

    def apply(self, x):
        y = np.empty(self.n)
        xc = np.ascontiguousarray(x, np.float64)  # kept alive across the call
        lib().ref_fsai_apply(self.h, _p(xc), _p(y))
        return y

    def __del__(self):
        if getattr(self, "h", None):
            lib().ref_fsai_destroy(self.h)
            self.h = None


class Cpr:
    """CPR<int,int,double,FSAI,FSAI> of precond/CPR.hpp:42-172 (mutates copies of A, b)."""

    def __init__(self, params: dict | str, r, c, v, b):
        text = params if isinstance(params, str) else json.dumps(params)
        self.n = len(r) - 1
        self.h = lib().ref_cpr_create(text.encode(), self.n, _p(r), _p(c), _p(v), _p(b))
        self.setup_time = lib().ref_cpr_setup_time(self.h)
        sz = np.zeros(5, np.int64)
        lib().ref_cpr_sizes(self.h, _p(sz))
        self.nnzA, self.np_, self.nnzAp, self.nnzFg, self.nnzFl = (int(t) for t in sz)

    def decoupled(self):
        n = self.n
        r = np.empty(n + 1, np.int32)
        c = np.empty(self.nnzA, np.int32)
        v = np.empty(self.nnzA)
        b = np.empty(n)
        lib().ref_cpr_get_A(self.h, _p(r), _p(c), _p(v), _p(b))
        return r, c, v, b

    def pressure(self):
        r = np.empty(self.np_ + 1, np.int32)
        c = np.empty(self.nnzAp, np.int32)
        v = np.empty(self.nnzAp)
        lib().ref_cpr_get_Ap(self.h, _p(r), _p(c), _p(v))
        return r, c, v

    def fsai(self, which):
        nz = self.nnzFg if which == 0 else self.nnzFl
        n = self.n if which == 0 else self.np_
        Lr, Ur = np.empty(n + 1, np.int32), np.empty(n + 1, np.int32)
        Lc, Uc = np.empty(nz, np.int32), np.empty(nz, np.int32)
        Lv, Uv = np.empty(nz), np.empty(nz)
        if lib().ref_cpr_get_fsai(self.h, which, _p(Lr), _p(Lc), _p(Lv), _p(Ur), _p(Uc), _p(Uv)) != 0:
            return None
        return (Lr, Lc, Lv), (Ur, Uc, Uv)

    def apply(self, rvec):
        x = np.zeros(self.n)
        rc = np.ascontiguousarray(rvec, np.float64)  # kept alive across the call
        lib().ref_cpr_apply(self.h, _p(rc), _p(x))
        return x

    def solve(self, sol: dict | str):
        text = sol if isinstance(sol, str) else json.dumps(sol)
        x = np.empty(self.n)
        it, fl = C.c_int(), C.c_int()
        ra, rr, ts = C.c_double(), C.c_double(), C.c_double()
        lib().ref_solve(self.h, text.encode(), _p(x), C.byref(it), C.byref(ra), C.byref(rr), C.byref(fl),
                        C.byref(ts))
        return dict(x=x, iter=it.value, res_abs=ra.value, res_rel=rr.value, flag=fl.value, time=ts.value)

    def __del__(self):
        if getattr(self, "h", None):
            lib().ref_cpr_destroy(self.h)
            self.h = None


def num_threads() -> int:
    return lib().ref_num_threads()
