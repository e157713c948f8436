import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the native libraries and the oracle once per session (no-op when up to date)."""
    from deco_b200 import build
    build.build_gen()
    from oracle import port, ref
    port.build() if not os.path.exists(port.LIB) else None
    if ref.REF_SRC and os.path.isdir(ref.REF_SRC):
        ref.build()
    yield


def cpr_json(bs, seq=3, drs=0, weights="quasiimpes_GE", glo_rel=0.0, glo_abs=1e-16, loc_rel=1e-4, loc_abs=1e-16,
             tol_zero=0.0, cpd=1, e_ps=0.0, glo="FSAI", loc="FSAI", glo_bs=None, loc_bs=None, glo_power=1,
             loc_power=1):
    """A `prec` object in the reference's parameter-file layout (precond/CPR.hpp:49-65,118,130);
    glo/loc "Jacobi" select Jacobi stages, glo_bs/loc_bs their block_size (Jacobi.hpp:21)."""
    g = {"type": glo, "tol_rel": str(glo_rel), "tol_abs": str(glo_abs), "power": str(glo_power)}
    l = {"type": loc, "tol_rel": str(loc_rel), "tol_abs": str(loc_abs), "power": str(loc_power)}
    if glo_bs is not None or seq == 2 or glo == "Jacobi":
        g["block_size"] = str(glo_bs if glo_bs is not None else bs)
    if loc_bs is not None or loc == "Jacobi":
        l["block_size"] = str(loc_bs if loc_bs is not None else 1)
    return {"type": "CPR", "block_size": str(bs), "pressure_id": "0", "seq": str(seq), "weights": weights,
            "use_drs": str(drs), "drs": {"e_dd": "0.2", "e_ps": str(e_ps)}, "CPD": str(cpd),
            "tol_zero": str(tol_zero), "prec_glo": g, "prec_loc": l}


def sol_json(type_="rgmres", reltol=1e-8, restart=50, itmax=3000):
    return {"type": type_, "reltol": str(reltol), "restart": str(restart), "itmax": str(itmax), "verbosity": "0"}


def rel(a, b):
    import numpy as np
    nb = float(np.linalg.norm(b))
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b))) / (nb if nb > 0 else 1.0)
