"""deco_b200 — B200-native CPR-Krylov path of the deco solver library.

Python mirror of the reference's host classes over the C ABI of
include/deco_b200.h (libdeco_b200.so).  Device memory is held in torch CUDA
tensors; the native library does all the work.

  CSR   core/CSR.hpp            device CSR<int,int,double>; apply(x, b, bs)
  FSAI  precond/FSAI/FSAI.hpp   FSAI(param, A); apply(x, b) (x may be b)
  CPR   precond/CPR.hpp         CPR(prec, A, b) mutates A and b; apply(r, x)
  SOL   solver/SOL.hpp          SOL(sol, A, precond, b, x=None) solves in the constructor
  ADJ   (no reference counterpart) adjoint of the solve: A^T lambda = g with CPR on A^T;
        deco_b200.adjoint wraps forward + adjoint as a torch.autograd.Function
  Batch (no reference counterpart) many systems x several right-hand sides in one lockstep solve

Parameter dictionaries use the reference's JSON keys (values may be strings, as
in the shipped param_*.json files).
"""
from __future__ import annotations

import ctypes as C
import json

import numpy as np

from ._lib import BatchResult, CprParams, DecoError, SolParams, SolResult, check, lib

__all__ = ["Context", "CSR", "FSAI", "CPR", "SOL", "ADJ", "Batch", "DecoError", "default_context", "load_params",
           "cpr_params", "sol_params"]

_WEIGHTS = {"none": 0, "quasiimpes": 1, "quasiimpes_GE": 2}
_SOLVERS = {"rgmres": 0, "lgmres": 1}


def _torch():
    import torch
    return torch


def _ptr(t):
    return C.c_void_p(t.data_ptr())


class Context:
    """Device + stream (replaces the reference's global MPI communicator and
    OpenMP pool).  Uses torch's current stream so torch ops and library calls
    are ordered."""

    def __init__(self, device: int = 0, stream=None):
        torch = _torch()
        if not torch.cuda.is_available():
            raise DecoError(-2, "no CUDA device available: the deco_b200 path has no CPU fallback")
        torch.cuda.set_device(device)
        self.device = device
        if stream is None:
            stream = torch.cuda.current_stream(device)
            if stream.cuda_stream == 0:
                # the legacy default stream has no handle to share: give the library and
                # torch one common stream so their work stays ordered
                stream = torch.cuda.Stream(device)
                torch.cuda.set_stream(stream)
        self.torch_stream = stream
        h = C.c_void_p()
        check(lib().deco_ctx_create(device, C.c_void_p(self.torch_stream.cuda_stream), C.byref(h)))
        self.h = h

    def sync(self):
        check(lib().deco_ctx_sync(self.h))

    def set_autotune(self, on: bool):
        check(lib().deco_ctx_set_autotune(self.h, int(on)))

    def trim(self):
        """Returns the library's cached device blocks to the device memory pool."""
        check(lib().deco_ctx_trim(self.h))

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().deco_ctx_destroy(self.h)
                self.h = None
        except Exception:  # interpreter shutdown: the binding may already be gone
            pass


_default = None


def default_context() -> Context:
    global _default
    if _default is None:
        _default = Context(0)
    return _default


def _dev(t, dtype):
    torch = _torch()
    if isinstance(t, np.ndarray):
        t = torch.from_numpy(np.ascontiguousarray(t))
    return t.to(device="cuda", dtype=dtype).contiguous()


class CSR:
    """CSR<int,int,double> on the device (core/CSR.hpp:4-13)."""

    def __init__(self, n, m, r, c, v, ctx: Context | None = None, _handle=None):
        self.ctx = ctx or default_context()
        self._borrowed = _handle is not None
        if _handle is not None:
            self.h = _handle
        elif hasattr(r, "data_ptr"):
            # torch tensors: device arrays (copied on the device) or (pinned) host arrays
            torch = _torch()
            assert r.dtype == torch.int32 and c.dtype == torch.int32 and v.dtype == torch.float64
            assert r.is_contiguous() and c.is_contiguous() and v.is_contiguous()
            where = 1 if r.is_cuda else 0
            h = C.c_void_p()
            check(lib().deco_csr_create(self.ctx.h, int(n), int(m), int(c.numel()), C.c_void_p(r.data_ptr()),
                                        C.c_void_p(c.data_ptr()), C.c_void_p(v.data_ptr()), where, C.byref(h)))
            self.h = h
        else:
            r = np.ascontiguousarray(r, np.int32)
            c = np.ascontiguousarray(c, np.int32)
            v = np.ascontiguousarray(v, np.float64)
            h = C.c_void_p()
            check(lib().deco_csr_create(self.ctx.h, int(n), int(m), int(len(c)), r.ctypes.data, c.ctypes.data,
                                        v.ctypes.data, 0, C.byref(h)))
            self.h = h
        n_, m_, nz_ = C.c_int(), C.c_int(), C.c_int()
        check(lib().deco_csr_info(self.h, C.byref(n_), C.byref(m_), C.byref(nz_)))
        self.n, self.m = n_.value, m_.value

    @property
    def nz(self) -> int:
        n_, m_, nz_ = C.c_int(), C.c_int(), C.c_int()
        check(lib().deco_csr_info(self.h, C.byref(n_), C.byref(m_), C.byref(nz_)))
        return nz_.value

    @classmethod
    def from_system(cls, sysm, ctx=None):
        return cls(sysm.n, sysm.n, sysm.r, sysm.c, sysm.v, ctx)

    def apply(self, x, b=None, bs: int = 1):
        """b = A x (bs == 1) or the restricted product of alg::spmv (bs > 1)."""
        torch = _torch()
        x = _dev(x, torch.float64)
        if b is None:
            b = torch.empty((self.n + bs - 1) // bs, dtype=torch.float64, device="cuda")
        check(lib().deco_spmv(self.ctx.h, self.h, _ptr(x), _ptr(b), bs))
        return b

    def apply_f32(self, x, b=None, bs: int = 1):
        torch = _torch()
        if not getattr(self, "_f32_ready", False):
            check(lib().deco_csr_make_f32(self.ctx.h, self.h))
            self._f32_ready = True
        x = _dev(x, torch.float32)
        if b is None:
            b = torch.empty((self.n + bs - 1) // bs, dtype=torch.float32, device="cuda")
        check(lib().deco_spmv_f32(self.ctx.h, self.h, _ptr(x), _ptr(b), bs))
        return b

    def residual(self, b, x, r=None):
        torch = _torch()
        if r is None:
            r = torch.empty(self.n, dtype=torch.float64, device="cuda")
        check(lib().deco_residual(self.ctx.h, self.h, _ptr(b), _ptr(x), _ptr(r)))
        return r

    def download(self):
        nz = self.nz
        r = np.empty(self.n + 1, np.int32)
        c = np.empty(nz, np.int32)
        v = np.empty(nz, np.float64)
        check(lib().deco_csr_download(self.ctx.h, self.h, r.ctypes.data, c.ctypes.data, v.ctypes.data))
        return r, c, v

    def set_values(self, v):
        if hasattr(v, "data_ptr"):
            torch = _torch()
            assert v.dtype == torch.float64 and v.is_contiguous() and v.numel() == self.nz
            check(lib().deco_csr_set_values(self.ctx.h, self.h, _ptr(v), 1 if v.is_cuda else 0))
            return
        v = np.ascontiguousarray(v, np.float64)
        check(lib().deco_csr_set_values(self.ctx.h, self.h, v.ctypes.data, 0))

    def set_blocks(self, bs: int):
        """Adds (bs 2 or 3) or removes (0) the cell-block copy used by later products."""
        check(lib().deco_csr_set_blocks(self.ctx.h, self.h, int(bs)))

    @property
    def blocks(self):
        """(block size, stored blocks) of the cell-block copy; (0, 0) without one."""
        b, k = C.c_int(), C.c_int()
        check(lib().deco_csr_blocks(self.h, C.byref(b), C.byref(k)))
        return b.value, k.value

    @property
    def padded(self):
        """Slots per cell (or row) of the padded copy the products use (4, 7 or 8; 0: none)."""
        w = C.c_int()
        check(lib().deco_csr_padded(self.h, C.byref(w)))
        return w.value

    def product_plan(self, precision: int = 64):
        """(kind, lanes) of the product y = A x takes: kind "padded" (rows grouped per
        thread), "cells" (lanes per cell) or "csr" (lanes per row), as the
        autotuner of a CPR setup chose it, or the layout rules."""
        k, w = C.c_int(), C.c_int()
        check(lib().deco_csr_product_plan(self.h, precision, C.byref(k), C.byref(w)))
        return {1: "padded", 2: "cells", 3: "csr"}[k.value], w.value

    @property
    def slot_codes(self):
        """(bytes per slot column the padded products read: 1, 2 or 4, 0 without a
        padded copy; distinct column offsets the codes select)."""
        b, k = C.c_int(), C.c_int()
        check(lib().deco_csr_slot_codes(self.h, C.byref(b), C.byref(k)))
        return b.value, k.value

    def transpose(self) -> "CSR":
        """A^T on the device, rows in ascending column order."""
        h = C.c_void_p()
        check(lib().deco_csr_transpose(self.ctx.h, self.h, C.byref(h)))
        T = CSR(0, 0, None, None, None, ctx=self.ctx, _handle=h)
        T._borrowed = False
        return T

    def grad_pattern(self, lam, x, alpha: float = -1.0, out=None):
        """out[e] = alpha * lam[i] * x[j] for every stored entry e = (i, j): dL/dA for alpha = -1."""
        torch = _torch()
        lam = _dev(lam, torch.float64)
        x = _dev(x, torch.float64)
        if out is None:
            out = torch.empty(self.nz, dtype=torch.float64, device="cuda")
        check(lib().deco_grad_A_pattern(self.ctx.h, self.h, _ptr(lam), _ptr(x), float(alpha), _ptr(out)))
        return out

    @property
    def subwarp(self) -> int:
        s = C.c_int()
        check(lib().deco_csr_subwarp(self.h, C.byref(s)))
        return s.value

    @subwarp.setter
    def subwarp(self, sw: int):
        check(lib().deco_csr_set_subwarp(self.h, int(sw)))

    def __del__(self):
        if getattr(self, "h", None) and not self._borrowed:
            lib().deco_csr_destroy(self.h)
            self.h = None


class FSAI:
    """FSAI(const ptree&, shared_ptr<CSR>) of precond/FSAI/FSAI.hpp:14-37."""

    def __init__(self, param: dict | None, A: CSR | None, precision: int = 64, _handle=None, _owner=None):
        self._owner = _owner
        if _handle is not None:
            self.ctx = _owner.ctx
            self.h = _handle
            self._borrowed = True
        else:
            self.ctx = A.ctx
            self._borrowed = False
            p = param or {}
            h = C.c_void_p()
            check(lib().deco_fsai_create(self.ctx.h, A.h, float(p.get("tol_rel", 0.0)), float(p.get("tol_abs", 0.0)),
                                         int(p.get("power", 1)), int(precision), C.byref(h)))
            self.h = h
        n, nz, k = C.c_int(), C.c_int(), C.c_int()
        check(lib().deco_fsai_info(self.h, C.byref(n), C.byref(nz), C.byref(k)))
        self.n, self.nz, self.max_order = n.value, nz.value, k.value

    def apply(self, x, b=None):
        torch = _torch()
        x = _dev(x, torch.float64)
        if b is None:
            b = torch.empty(self.n, dtype=torch.float64, device="cuda")
        check(lib().deco_fsai_apply(self.ctx.h, self.h, _ptr(x), _ptr(b)))
        return b

    def apply_f32(self, x, b=None):
        """b = FU^T (FL x) in float32 vectors (a factor made with precision 32)."""
        torch = _torch()
        x = _dev(x, torch.float32)
        if b is None:
            b = torch.empty(self.n, dtype=torch.float32, device="cuda")
        check(lib().deco_fsai_apply_f32(self.ctx.h, self.h, _ptr(x), _ptr(b)))
        return b

    @property
    def padded(self):
        """(slots of FL's, slots of FU^T's) padded copies (4, 7 or 8; 0 without)."""
        a, b = C.c_int(), C.c_int()
        check(lib().deco_fsai_padded(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    @property
    def slot_codes(self):
        """Bytes per slot column of FL's and FU^T's padded copies (1, 2 or 4; 0 without)."""
        a, b = C.c_int(), C.c_int()
        check(lib().deco_fsai_slot_codes(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    @property
    def blocks(self):
        """(block size, stored blocks of FL, stored blocks of FU^T); block size 0 without block copies."""
        b, kl, ku = C.c_int(), C.c_int(), C.c_int()
        check(lib().deco_fsai_blocks(self.h, C.byref(b), C.byref(kl), C.byref(ku)))
        return b.value, kl.value, ku.value

    def factors(self):
        n, nz = self.n, self.nz
        Lr, Ur = np.empty(n + 1, np.int32), np.empty(n + 1, np.int32)
        Lc, Uc = np.empty(nz, np.int32), np.empty(nz, np.int32)
        Lv, Uv = np.empty(nz), np.empty(nz)
        check(lib().deco_fsai_download(self.ctx.h, self.h, Lr.ctypes.data, Lc.ctypes.data, Lv.ctypes.data,
                                       Ur.ctypes.data, Uc.ctypes.data, Uv.ctypes.data))
        return (Lr, Lc, Lv), (Ur, Uc, Uv)

    def __del__(self):
        if getattr(self, "h", None) and not self._borrowed:
            lib().deco_fsai_destroy(self.h)
            self.h = None


def load_params(path_or_text: str) -> dict:
    """Reads a reference parameter file (// and /* */ comments allowed, IO/ptree.hpp:27-84)."""
    import re
    text = path_or_text
    if not text.lstrip().startswith("{"):
        with open(path_or_text) as f:
            text = f.read()
    out_lines = []
    in_block = False
    for line in text.splitlines():
        kept, pos = "", 0
        while pos < len(line):
            if in_block:
                e = line.find("*/", pos)
                if e < 0:
                    break
                in_block, pos = False, e + 2
                continue
            sl, ml = line.find("//", pos), line.find("/*", pos)
            if sl >= 0 and (ml < 0 or sl < ml):
                kept += line[pos:sl]
                break
            if ml >= 0:
                kept += line[pos:ml]
                e = line.find("*/", ml + 2)
                if e < 0:
                    in_block = True
                    break
                pos = e + 2
                continue
            kept += line[pos:]
            break
        if kept.strip():
            out_lines.append(kept)
    del re
    return json.loads("\n".join(out_lines))


def cpr_params(prec: dict, precision: int = 64) -> CprParams:
    """The `prec` object of a parameter file -> deco_cpr_params (precond/CPR.hpp:49-65,118,130)."""
    g, l = prec.get("prec_glo", {}), prec.get("prec_loc", {})
    drs = prec.get("drs", {})
    return CprParams(
        block_size=int(prec["block_size"]), pressure_id=int(prec.get("pressure_id", 0)), seq=int(prec.get("seq", 3)),
        weights=_WEIGHTS[prec.get("weights", "quasiimpes_GE")], use_drs=int(prec.get("use_drs", 0)),
        drs_e_dd=float(drs.get("e_dd", 0.2)), drs_e_ps=float(drs.get("e_ps", 0.0)), cpd=int(prec.get("CPD", 1)),
        tol_zero=float(prec.get("tol_zero", 0.0)), glo_tol_rel=float(g.get("tol_rel", 0.0)),
        glo_tol_abs=float(g.get("tol_abs", 0.0)), glo_power=int(g.get("power", 1)),
        loc_tol_rel=float(l.get("tol_rel", 0.0)), loc_tol_abs=float(l.get("tol_abs", 0.0)),
        loc_power=int(l.get("power", 1)), precision=int(precision), glo_type=_stage(g.get("type", "FSAI")),
        loc_type=_stage(l.get("type", "FSAI")), glo_block_size=int(g.get("block_size", prec["block_size"])),
        loc_block_size=int(l.get("block_size", 1)))


def _stage(t: str) -> int:
    if t == "FSAI":
        return 0
    if t == "Jacobi":
        return 1
    raise DecoError(-6, f"the GPU path builds FSAI or Jacobi stages (got {t}); hypre AMG stays on the CPU build")


def sol_params(sol: dict, precision: int = 64, use_x0: bool = False) -> SolParams:
    """The `sol` object of a parameter file -> deco_sol_params (solver/rgmres.tpp:13-16)."""
    t = sol.get("type", "rgmres")
    if t not in _SOLVERS:
        raise DecoError(-6, f"Invalid solver type: {t}")
    return SolParams(type=_SOLVERS[t], reltol=float(sol["reltol"]), restart=int(sol["restart"]),
                     itmax=int(sol["itmax"]), verbosity=int(sol.get("verbosity", 0)), precision=int(precision),
                     use_x0=int(use_x0))


class CPR:
    """CPR<int,int,double,FSAI,FSAI>(prec, A, b) of precond/CPR.hpp:42-172.
    A (CSR) and b (CUDA float64 tensor) are modified in place like the reference's."""

    def __init__(self, prec: dict, A: CSR, b, precision: int = 64):
        torch = _torch()
        if not (hasattr(b, "is_cuda") and b.is_cuda and b.dtype == torch.float64):
            raise DecoError(-1, "b must be a CUDA float64 tensor (it is decoupled in place)")
        self.A, self.b, self.ctx = A, b, A.ctx
        self.params = cpr_params(prec, precision)
        h = C.c_void_p()
        check(lib().deco_cpr_create(self.ctx.h, A.h, _ptr(b), C.byref(self.params), C.byref(h)))
        self.h = h
        self.n = A.n

    @property
    def Ap(self) -> CSR:
        """The pressure matrix A_pp (borrowed: the returned object keeps this CPR alive;
        the CPR holds no reference back, so dropping the CPR frees its device memory at once)."""
        hp = C.c_void_p()
        check(lib().deco_cpr_pressure(self.h, C.byref(hp)))
        M = CSR(0, 0, None, None, None, ctx=self.ctx, _handle=hp)
        M._owner = self
        return M

    def fsai(self, which: int) -> FSAI:
        hf = C.c_void_p()
        check(lib().deco_cpr_fsai(self.h, which, C.byref(hf)))
        return FSAI(None, None, _handle=hf, _owner=self)

    def apply(self, r, x=None):
        torch = _torch()
        r = _dev(r, torch.float64)
        if x is None:
            x = torch.empty(self.n, dtype=torch.float64, device="cuda")
        check(lib().deco_cpr_apply(self.ctx.h, self.h, _ptr(r), _ptr(x)))
        return x

    def decouple_rhs(self, b):
        """Decouples another right-hand side in place, bit-identically to the b given at setup."""
        torch = _torch()
        if not (hasattr(b, "is_cuda") and b.is_cuda and b.dtype == torch.float64 and b.is_contiguous()):
            raise DecoError(-1, "b must be a contiguous CUDA float64 tensor (it is decoupled in place)")
        check(lib().deco_cpr_decouple_rhs(self.ctx.h, self.h, _ptr(b)))
        return b

    def timings(self) -> dict:
        t = (C.c_double * 5)()
        check(lib().deco_cpr_timings(self.h, t))
        return dict(zip(["decoupling", "get local matrix", "Global precond", "Local  precond", "Prec"], list(t)))

    @property
    def fixed_diagonals(self) -> int:
        k = C.c_int()
        check(lib().deco_cpr_fixed_diagonals(self.h, C.byref(k)))
        return k.value

    def __del__(self):
        if getattr(self, "h", None):
            lib().deco_cpr_destroy(self.h)
            self.h = None


class SOL:
    """SOL<R,C,V>(sol, A, precond, b, x) of solver/SOL.hpp:19-39: the solve runs in
    the constructor; results in x, iter, res_abs, res_rel, flag (+ resvec), and
    res_rel_orig, the relative residual of the original system before the CPR
    decoupling (res_rel is on the decoupled system, as in the reference)."""

    def __init__(self, sol: dict, A: CSR, precond: CPR | None, b, x=None, precision: int = 64):
        torch = _torch()
        self.params = sol_params(sol, precision, use_x0=x is not None)
        self.ctx = A.ctx
        b = _dev(b, torch.float64)
        self.x = x if x is not None else torch.zeros(A.n, dtype=torch.float64, device="cuda")
        res = SolResult()
        self.resvec = np.zeros(max(self.params.itmax, 0) + 1)
        check(lib().deco_gmres_solve(self.ctx.h, A.h, precond.h if precond is not None else None, _ptr(b),
                                     _ptr(self.x), C.byref(self.params), C.byref(res), self.resvec.ctypes.data))
        self.iter, self.flag = res.iter, res.flag
        self.res_abs, self.res_rel = res.res_abs, res.res_rel
        self.res_rel_orig = res.res_rel_orig
        self.time_ms, self.restarts = res.t_solve_ms, res.restarts
        self.phases_ms = {"precond": res.t_precond_ms, "matvec": res.t_matvec_ms, "ortho": res.t_ortho_ms,
                          "dots": res.t_dots_ms}
        self.resvec = self.resvec[: self.iter]

    def get_result(self):
        return self.x


class ADJ:
    """Adjoint of the CPR-GMRES solve (no counterpart in the reference).

    ``ADJ(prec, A)`` transposes A (its current values: build it before any forward
    decoupling) and sets up CPR on A^T; ``solve(sol, g)`` returns lambda with
    A^T lambda = g.  dL/db = lambda; dL/dA on A's pattern is
    ``A.grad_pattern(lambda, x)``."""

    def __init__(self, prec: dict, A: CSR, precision: int = 64):
        self.ctx = A.ctx
        self.n = A.n
        self.params = cpr_params(prec, precision)
        h = C.c_void_p()
        check(lib().deco_adjoint_create(self.ctx.h, A.h, C.byref(self.params), C.byref(h)))
        self.h = h

    def solve(self, sol: dict, g, lam=None, precision: int | None = None):
        torch = _torch()
        prec = self.params.precision if precision is None else precision
        sp = sol_params(sol, prec, use_x0=lam is not None)
        g = _dev(g, torch.float64)
        if lam is None:
            lam = torch.zeros(self.n, dtype=torch.float64, device="cuda")
        res = SolResult()
        self.resvec = np.zeros(max(sp.itmax, 0) + 1)
        check(lib().deco_adjoint_solve(self.ctx.h, self.h, _ptr(g), _ptr(lam), C.byref(sp), C.byref(res),
                                       self.resvec.ctypes.data))
        self.iter, self.flag = res.iter, res.flag
        self.res_abs, self.res_rel = res.res_abs, res.res_rel
        self.res_rel_orig = res.res_rel_orig
        self.time_ms = res.t_solve_ms
        self.resvec = self.resvec[: self.iter]
        return lam

    def transposed(self) -> CSR:
        """A^T as decoupled by the adjoint's CPR (owned by this object)."""
        h = C.c_void_p()
        check(lib().deco_adjoint_parts(self.h, C.byref(h), None))
        T = CSR(0, 0, None, None, None, ctx=self.ctx, _handle=h)
        T._owner = self
        return T

    def __del__(self):
        if getattr(self, "h", None):
            lib().deco_adjoint_destroy(self.h)
            self.h = None


class Batch:
    """Independent systems, each with `nrhs` right-hand sides, solved together (no
    counterpart in the reference).  A: the block-diagonal matrix of all systems
    (decoupled in place, as CPR does); row_off: nsys + 1 cell-aligned row offsets.
    Right-hand sides and solutions are row-interleaved: B[row * nrhs + k]."""

    def __init__(self, prec: dict, A: CSR, row_off, nrhs: int, precision: int = 64):
        self.ctx, self.A, self.n = A.ctx, A, A.n
        self.row_off = np.ascontiguousarray(row_off, np.int32)
        self.nsys, self.nrhs = len(self.row_off) - 1, int(nrhs)
        self.params = cpr_params(prec, precision)
        h = C.c_void_p()
        check(lib().deco_batch_create(self.ctx.h, A.h, self.nsys, self.row_off.ctypes.data, self.nrhs,
                                      C.byref(self.params), C.byref(h)))
        self.h = h

    @property
    def widths(self) -> np.ndarray:
        w = np.zeros(self.nsys, np.int32)
        check(lib().deco_batch_info(self.h, None, None, None, w.ctypes.data))
        return w

    def apply(self, R, X=None):
        """X = M^{-1} R for every column (the batch's CPR; row-interleaved multi-vectors)."""
        torch = _torch()
        R = _dev(R, torch.float64)
        if X is None:
            X = torch.empty(self.n * self.nrhs, dtype=torch.float64, device="cuda")
        check(lib().deco_batch_apply(self.ctx.h, self.h, _ptr(R), _ptr(X)))
        return X

    def cpr(self):
        """The batch's CPR (a borrowed handle; single-vector apply on the whole block-diagonal system)."""
        h = C.c_void_p()
        check(lib().deco_batch_cpr(self.h, C.byref(h)))
        return h

    def solve(self, sol: dict, B, X=None):
        """X (CUDA float64, n * nrhs) solving every system for every column of B."""
        torch = _torch()
        B = _dev(B, torch.float64)
        if X is None:
            X = torch.empty(self.n * self.nrhs, dtype=torch.float64, device="cuda")
        sp = sol_params(sol, self.params.precision)
        q = self.nsys * self.nrhs
        it = np.zeros(q, np.int32)
        rr = np.zeros(q, np.float64)
        fl = np.zeros(q, np.int32)
        res = BatchResult()
        check(lib().deco_batch_solve(self.ctx.h, self.h, _ptr(B), _ptr(X), C.byref(sp), it.ctypes.data,
                                     rr.ctypes.data, fl.ctypes.data, C.byref(res)))
        self.iters = it.reshape(self.nsys, self.nrhs)
        self.res_rel = rr.reshape(self.nsys, self.nrhs)
        self.flags = fl.reshape(self.nsys, self.nrhs)
        self.result = {"max_iter": res.max_iter, "converged": res.converged, "cycles": res.cycles,
                       "graph": int(res.graph), "t_solve_ms": res.t_solve_ms}
        return X

    def __del__(self):
        if getattr(self, "h", None):
            lib().deco_batch_destroy(self.h)
            self.h = None
