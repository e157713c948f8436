"""FP64 CPU reference gradient of the CPR-GMRES solve x = A^{-1} b.

TEST INFRASTRUCTURE ONLY — used by tests/ as the checker of the GPU adjoint;
never by the product.

The reference solves forward only (solver/SOL.hpp:19-39); this module states the
adjoint mathematics the GPU path implements and evaluates it with the
reference's own CPR-GMRES (oracle/_ref, impl="ref") or the C restatement
(oracle/port.py, impl="port"):

    forward   A x = b                 CPR built on A (precond/CPR.hpp:42-172)
    adjoint   A^T lam = g,  g = dL/dx CPR built on A^T: transposed, then decoupled
    dL/db   = lam
    dL/dA_ij = -lam_i x_j             on A's sparsity pattern only

Both solves run in float64 with rgmres (solver/rgmres.tpp:8-139).  Decoupling
is a left multiplication by a block-diagonal matrix, so the GMRES solution of
the decoupled transposed system is lam itself.
"""
from __future__ import annotations

import numpy as np


def transpose(r, c, v, m: int | None = None):
    """CSR transpose with every row in ascending column order."""
    r = np.asarray(r, np.int64)
    c = np.asarray(c, np.int64)
    n = len(r) - 1
    m = int(c.max()) + 1 if m is None and len(c) else (m or 0)
    rows = np.repeat(np.arange(n), np.diff(r))
    order = np.lexsort((rows, c))  # by column, then by source row
    cnt = np.bincount(c, minlength=m)
    rt = np.zeros(m + 1, np.int32)
    np.cumsum(cnt, out=rt[1:])
    return rt, rows[order].astype(np.int32), np.asarray(v, np.float64)[order]


def _solver(impl):
    if impl == "ref":
        from . import ref

        def run(prec, sol, r, c, v, b):
            return ref.Cpr({"prec": prec}, r, c, v, b.copy()).solve(sol)
        return run
    if impl == "port":
        from . import port

        def run(prec, sol, r, c, v, b):
            return port.Cpr(prec, r, c, v, b.copy()).solve(sol)
        return run
    raise ValueError(impl)


def solve(prec: dict, sol: dict, r, c, v, b, impl: str = "ref") -> dict:
    """x = A^{-1} b by CPR-GMRES (A, b are not modified)."""
    return _solver(impl)(prec, sol, np.asarray(r, np.int32), np.asarray(c, np.int32),
                         np.asarray(v, np.float64).copy(), np.asarray(b, np.float64))


def adjoint(prec: dict, sol: dict, r, c, v, g, impl: str = "ref") -> dict:
    """lam = A^{-T} g with CPR on the transposed system."""
    rt, ct, vt = transpose(r, c, v, len(r) - 1)
    return _solver(impl)(prec, sol, rt, ct, vt, np.asarray(g, np.float64))


def grad_pattern(r, c, lam, x, alpha: float = -1.0):
    """alpha * lam_i * x_j for every stored entry (i, j), in CSR order."""
    rows = np.repeat(np.arange(len(r) - 1), np.diff(r))
    return alpha * (np.asarray(lam)[rows] * np.asarray(x)[np.asarray(c)])


def gradient(prec: dict, sol: dict, r, c, v, b, g, impl: str = "ref"):
    """(x, lam, dL/dA on A's pattern, forward info, adjoint info) for dL/dx = g."""
    fwd = solve(prec, sol, r, c, v, b, impl)
    adj = adjoint(prec, sol, r, c, v, g, impl)
    return fwd["x"], adj["x"], grad_pattern(r, c, adj["x"], fwd["x"]), fwd, adj
