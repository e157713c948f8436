"""ctypes binding of libdeco_gen.so (include/deco_gen.h): seeded synthetic systems."""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))


class GenParams(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("bs", C.c_int),
        ("sigma", C.c_double), ("kz_kx", C.c_double), ("layered", C.c_int),
        ("n_channels", C.c_int), ("channel_contrast", C.c_double), ("fault_frac", C.c_double),
        ("n_wells", C.c_int), ("acc_lo", C.c_double), ("acc_hi", C.c_double),
        ("cpl_lo", C.c_double), ("cpl_hi", C.c_double), ("comp", C.c_double),
        ("smooth", C.c_int), ("seed", C.c_ulonglong),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(_PKG, "libdeco_gen.so")
        if not os.path.exists(path):
            from . import build
            build.build_gen()
        L = C.CDLL(path)
        L.deco_gen_preset.argtypes = [C.c_int, C.c_ulonglong, C.POINTER(GenParams)]
        L.deco_gen_size.argtypes = [C.POINTER(GenParams), C.POINTER(C.c_int), C.POINTER(C.c_longlong)]
        L.deco_gen_fill.argtypes = [C.POINTER(GenParams), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_void_p]
        L.deco_gen_fill_logk.argtypes = [C.POINTER(GenParams), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_void_p]
        L.deco_gen_grad_logk.argtypes = [C.POINTER(GenParams), C.c_void_p, C.c_void_p, C.c_void_p]
        L.deco_gen_uniform.argtypes = [C.c_ulonglong, C.c_ulonglong, C.c_longlong, C.c_void_p]
        L.deco_gen_uniform.restype = None
        _lib = L
    return _lib


@dataclass
class System:
    """A CSR system A x = b (reference layout: core/CSR.hpp:4-13)."""
    n: int
    r: np.ndarray  # int32[n+1]
    c: np.ndarray  # int32[nnz]
    v: np.ndarray  # float64[nnz]
    b: np.ndarray  # float64[n]
    bs: int
    params: GenParams
    logk: np.ndarray | None = None

    @property
    def nnz(self) -> int:
        return int(self.r[-1])


def preset(config: int, seed: int = 1234, **overrides) -> GenParams:
    p = GenParams()
    if lib().deco_gen_preset(config, seed, C.byref(p)) != 0:
        raise ValueError(f"unknown preset {config}")
    for k, val in overrides.items():
        setattr(p, k, val)
    return p


def generate(p: GenParams, with_logk: bool = False) -> System:
    n = C.c_int()
    nnz = C.c_longlong()
    rc = lib().deco_gen_size(C.byref(p), C.byref(n), C.byref(nnz))
    if rc != 0:
        raise ValueError(f"deco_gen_size failed ({rc})")
    r = np.empty(n.value + 1, np.int32)
    c = np.empty(nnz.value, np.int32)
    v = np.empty(nnz.value, np.float64)
    b = np.empty(n.value, np.float64)
    nc = p.nx * p.ny * p.nz
    logk = np.empty(nc, np.float64) if with_logk else None
    rc = lib().deco_gen_fill(C.byref(p), r.ctypes.data, c.ctypes.data, v.ctypes.data, b.ctypes.data,
                             logk.ctypes.data if logk is not None else None)
    if rc != 0:
        raise ValueError(f"deco_gen_fill failed ({rc})")
    return System(n.value, r, c, v, b, p.bs, p, logk)


def generate_from_logk(p: GenParams, logk: np.ndarray) -> System:
    """The system of preset ``p`` with the permeability field ``exp(logk)`` (one value per cell)."""
    n = C.c_int()
    nnz = C.c_longlong()
    if lib().deco_gen_size(C.byref(p), C.byref(n), C.byref(nnz)) != 0:
        raise ValueError("deco_gen_size failed")
    logk = np.ascontiguousarray(logk, np.float64)
    if logk.size != p.nx * p.ny * p.nz:
        raise ValueError("logk needs one value per cell")
    r = np.empty(n.value + 1, np.int32)
    c = np.empty(nnz.value, np.int32)
    v = np.empty(nnz.value, np.float64)
    b = np.empty(n.value, np.float64)
    rc = lib().deco_gen_fill_logk(C.byref(p), logk.ctypes.data, r.ctypes.data, c.ctypes.data, v.ctypes.data,
                                  b.ctypes.data)
    if rc != 0:
        raise ValueError(f"deco_gen_fill_logk failed ({rc})")
    return System(n.value, r, c, v, b, p.bs, p, logk.copy())


def grad_logk(p: GenParams, logk: np.ndarray | None, dLdA: np.ndarray) -> np.ndarray:
    """dL/d ln k per cell from dL/dA given on the pattern of the system of ``p`` (chain rule through the
    harmonic-mean transmissibilities)."""
    dLdA = np.ascontiguousarray(dLdA, np.float64)
    out = np.empty(p.nx * p.ny * p.nz, np.float64)
    if logk is not None:
        logk = np.ascontiguousarray(logk, np.float64)
        if logk.size != out.size:
            raise ValueError("logk needs one value per cell")
    rc = lib().deco_gen_grad_logk(C.byref(p), logk.ctypes.data if logk is not None else None, dLdA.ctypes.data,
                                  out.ctypes.data)
    if rc != 0:
        raise ValueError(f"deco_gen_grad_logk failed ({rc})")
    return out


def uniform(seed: int, stream: int, n: int) -> np.ndarray:
    out = np.empty(n, np.float64)
    lib().deco_gen_uniform(seed, stream, n, out.ctypes.data)
    return out


def grid(nx: int, ny: int, nz: int, bs: int = 2, seed: int = 1234, **kw) -> System:
    """Small custom grid with the value distributions of preset 1 (for tests)."""
    p = preset(1, seed)
    p.nx, p.ny, p.nz, p.bs = nx, ny, nz, bs
    for k, val in kw.items():
        setattr(p, k, val)
    return generate(p)


def batch(nsys: int = 64, seed: int = 1234, cells_lo: int = 10_000, cells_hi: int = 500_000, bs: int = 2,
          nrhs: int = 8):
    """Independent two-phase systems (the value distributions of preset 1) with cell
    counts drawn log-uniform in [cells_lo, cells_hi], concatenated into one
    block-diagonal CSR, plus `nrhs` uniform [0,1) right-hand sides per system
    (row-interleaved).  Returns (r, c, v, row_off, B, shapes)."""
    u = uniform(seed, 911, 2 * nsys)
    rs, cs, vs, offs, shapes = [], [], [], [0], []
    nz_off = 0
    for q in range(nsys):
        cells = float(np.exp(np.log(cells_lo) + u[q] * (np.log(cells_hi) - np.log(cells_lo))))
        nzc = max(2, int(round((cells / 4.0) ** (1.0 / 3.0))))  # nx = ny = 2 nz
        nxy = max(2, int(round(np.sqrt(cells / nzc))))
        p = preset(1, seed + 7919 * (q + 1))
        p.nx, p.ny, p.nz, p.bs = nxy, nxy, nzc, bs
        s = generate(p)
        shapes.append((nxy, nxy, nzc))
        rs.append(s.r[:-1] + nz_off)
        cs.append(s.c + offs[-1])
        vs.append(s.v)
        nz_off += s.nnz
        offs.append(offs[-1] + s.n)
    r = np.concatenate(rs + [np.array([nz_off], np.int64)]).astype(np.int32)
    c = np.concatenate(cs).astype(np.int32)
    v = np.concatenate(vs)
    row_off = np.array(offs, np.int32)
    n = int(row_off[-1])
    B = uniform(seed, 913, n * nrhs)
    return r, c, v, row_off, B, shapes


def batch_subset(r, c, v, row_off, B, nrhs: int, systems):
    """The block-diagonal matrix and right-hand sides of the listed systems of a batch
    (e.g. one rank's share when independent systems are spread over GPUs)."""
    rs, cs, vs, offs, bs_ = [], [], [], [0], []
    nz_off = 0
    Bm = np.asarray(B).reshape(-1, nrhs)
    for q in systems:
        a, e = int(row_off[q]), int(row_off[q + 1])
        ra, re = int(r[a]), int(r[e])
        rs.append((r[a:e] - ra + nz_off).astype(np.int64))
        cs.append(c[ra:re] - a + offs[-1])
        vs.append(v[ra:re])
        bs_.append(Bm[a:e])
        nz_off += re - ra
        offs.append(offs[-1] + (e - a))
    r2 = np.concatenate(rs + [np.array([nz_off], np.int64)]).astype(np.int32)
    return (r2, np.concatenate(cs).astype(np.int32), np.concatenate(vs), np.array(offs, np.int32),
            np.ascontiguousarray(np.concatenate(bs_).reshape(-1)))
