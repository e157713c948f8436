"""Generates the golden fixtures in this directory by running the REFERENCE's own
code (compiled from its sources into oracle/_ref by oracle/ref/Makefile) on small
seeded systems.  Each fixture stores its inputs, so it does not depend on the
generator staying unchanged.

    python tests/golden/make_golden.py

Stored per case (npz): the input CSR + b; the decoupled A and b after the CPR
constructor (precond/CPR.hpp:42-172); A_pp; both FSAI factors (FL lower, FU^T
upper; precond/FSAI/*); the CPR apply of a seeded vector; the restricted and
full SpMV of a seeded vector (core/alg.hpp:50-64); the rgmres and lgmres
iteration counts, residuals and solutions (solver/rgmres.tpp, lgmres.tpp).
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from conftest import cpr_json, sol_json  # noqa: E402
from deco_b200 import gen  # noqa: E402
from oracle import ref  # noqa: E402

CASES = {
    "tiny_bs2": (dict(nx=5, ny=4, nz=3, bs=2, seed=7), dict()),
    "small_bs3_drs": (dict(nx=6, ny=5, nz=4, bs=3, seed=11, fault_frac=0.03, layered=1, sigma=2.0, kz_kx=0.1),
                      dict(drs=1, glo_rel=0.2)),
    "small_bs2_seq1_qimpes": (dict(nx=8, ny=6, nz=3, bs=2, seed=13, n_channels=2, channel_contrast=1e3),
                              dict(seq=1, weights="quasiimpes")),
}


def make(name):
    gkw, pkw = CASES[name]
    g = dict(gkw)
    nx, ny, nz, bs, seed = g.pop("nx"), g.pop("ny"), g.pop("nz"), g.pop("bs"), g.pop("seed")
    s = gen.grid(nx, ny, nz, bs=bs, seed=seed, **g)
    prec = cpr_json(bs, **pkw)
    rng = np.random.default_rng(0)
    xv = rng.standard_normal(s.n)
    out = dict(r=s.r, c=s.c, v=s.v, b=s.b, xv=xv, bs=bs)
    out["spmv"] = ref.spmv(s.r, s.c, s.v, xv, 1)
    out["spmv_restricted"] = ref.spmv(s.r, s.c, s.v, xv, bs)
    R = ref.Cpr({"prec": prec}, s.r, s.c, s.v, s.b)
    out["Dr"], out["Dc"], out["Dv"], out["Db"] = R.decoupled()
    out["Pr"], out["Pc"], out["Pv"] = R.pressure()
    for w, tag in ((0, "G"), (1, "L")):
        (Lr, Lc, Lv), (Ur, Uc, Uv) = R.fsai(w)
        out.update({f"{tag}Lr": Lr, f"{tag}Lc": Lc, f"{tag}Lv": Lv, f"{tag}Ur": Ur, f"{tag}Uc": Uc, f"{tag}Uv": Uv})
    out["apply"] = R.apply(xv)
    for st in ("rgmres", "lgmres"):
        res = R.solve(sol_json(st, itmax=2000))
        out[f"{st}_iter"] = res["iter"]
        out[f"{st}_res_rel"] = res["res_rel"]
        out[f"{st}_flag"] = res["flag"]
        out[f"{st}_x"] = res["x"]
    out["prec_json"] = json.dumps(prec)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    return {k: (v.shape if hasattr(v, "shape") else v) for k, v in out.items() if k.endswith("iter")}


if __name__ == "__main__":
    if not ref.available() and not ref.build():
        sys.exit("oracle/_ref/libdeco_ref.so is not available")
    for nm in CASES:
        print(nm, make(nm))
