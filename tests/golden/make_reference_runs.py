"""Records the reference build's own CPR-GMRES runs on the benchmark systems.

    python tests/golden/make_reference_runs.py [config ...]     (default: 2 3)

For each seeded synthetic system (the generator presets of deco_b200.gen) it runs
the reference's CPR<FSAI,FSAI> setup and SOL::rgmres (oracle/_ref, compiled from
the reference's sources) with the benchmark's settings and writes what it
measured -- iteration count, relative residual, flag, setup and solve seconds,
OpenMP thread count -- to tests/golden/reference_runs.json.  bench.py reports
these iteration counts beside the GPU's (`reference_iterations`), and the GPU
tests compare against them where running the reference live would take
minutes.  The reference sums its dot products with `omp atomic`, so the count can
move by a few iterations with the thread count; the record says which was used.
"""
from __future__ import annotations

import json
import os
import platform
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

SEED = 1234
SOL = {"type": "rgmres", "reltol": "1e-8", "restart": "50", "itmax": "6000", "verbosity": "0"}


def prec_for(bs: int) -> dict:
    return {"type": "CPR", "block_size": str(bs), "pressure_id": "0", "seq": "3", "weights": "quasiimpes_GE",
            "use_drs": "0", "drs": {"e_dd": "0.2", "e_ps": "0.0"}, "CPD": "1", "tol_zero": "0.0",
            "prec_glo": {"type": "FSAI", "tol_rel": "0.0", "tol_abs": "1e-16", "power": "1"},
            "prec_loc": {"type": "FSAI", "tol_rel": "1e-4", "tol_abs": "1e-16", "power": "1"}}


def run(config: int) -> dict:
    import numpy as np
    from deco_b200 import gen
    from oracle import ref
    s = gen.generate(gen.preset(config, SEED))
    t0 = time.perf_counter()
    R = ref.Cpr({"prec": prec_for(s.bs)}, s.r, s.c, s.v, s.b)
    t_setup = time.perf_counter() - t0
    res = R.solve(SOL)
    Dr, Dc, Dv, Db = R.decoupled()
    true_rel = float(np.linalg.norm(Db - ref.spmv(Dr, Dc, Dv, res["x"])) / np.linalg.norm(Db))
    return {"config": config, "seed": SEED, "rows": s.n, "nnz": s.nnz, "bs": s.bs, "sol": SOL,
            "iterations": res["iter"], "res_rel": res["res_rel"], "true_rel_residual": true_rel, "flag": res["flag"],
            "setup_s": t_setup, "solve_s": res["time"], "omp_threads": ref.num_threads(),
            "host": platform.processor() or platform.machine()}


def main(argv):
    configs = [int(a) for a in argv] or [2, 3]
    path = os.path.join(HERE, "reference_runs.json")
    out = {}
    if os.path.exists(path):
        with open(path) as f:
            out = json.load(f)
    for c in configs:
        r = run(c)
        print(json.dumps(r), flush=True)
        out[f"config{c}"] = r
    with open(path, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
        f.write("\n")


if __name__ == "__main__":
    main(sys.argv[1:])
