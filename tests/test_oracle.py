"""Pins the CPU oracle (oracle/deco_oracle.c, the plain-C restatement) against
the reference: (1) the golden fixtures produced by the reference's own code
(tests/golden/make_golden.py), (2) the reference library built here, live, on
larger seeded systems.  CPU only."""
import glob
import json
import os

import numpy as np
import pytest

from conftest import cpr_json, rel, sol_json

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))


def test_golden_fixtures_present():
    assert len(GOLDEN) >= 3


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_port_reproduces_golden(path):
    from oracle import port
    g = np.load(path)
    prec = json.loads(str(g["prec_json"]))
    bs = int(g["bs"])
    assert rel(port.spmv(g["r"], g["c"], g["v"], g["xv"], 1), g["spmv"]) < 1e-15
    assert rel(port.spmv(g["r"], g["c"], g["v"], g["xv"], bs), g["spmv_restricted"]) < 1e-15
    O = port.Cpr(prec, g["r"], g["c"], g["v"], g["b"])
    Dr, Dc, Dv, Db = O.decoupled()
    for a, b in [(Dr, g["Dr"]), (Dc, g["Dc"])]:
        np.testing.assert_array_equal(a, b)
    if prec["weights"] == "quasiimpes":  # LAPACK dgesv rounding (CPR.hpp:364)
        assert rel(Dv, g["Dv"]) < 1e-14 and rel(Db, g["Db"]) < 1e-14
    else:
        np.testing.assert_array_equal(Dv, g["Dv"])
        np.testing.assert_array_equal(Db, g["Db"])
    Pr, Pc, Pv = O.pressure()
    np.testing.assert_array_equal(Pr, g["Pr"])
    np.testing.assert_array_equal(Pc, g["Pc"])
    assert rel(Pv, g["Pv"]) < 1e-14
    for w, tag in ((0, "G"), (1, "L")):
        (Lr, Lc, Lv), (Ur, Uc, Uv) = O.fsai(w)
        for a, b in [(Lr, g[tag + "Lr"]), (Lc, g[tag + "Lc"]), (Ur, g[tag + "Ur"]), (Uc, g[tag + "Uc"])]:
            np.testing.assert_array_equal(a, b)  # FSAI pattern: bit-exact
        assert rel(Lv, g[tag + "Lv"]) < 1e-13 and rel(Uv, g[tag + "Uv"]) < 1e-13
    assert rel(O.apply(g["xv"]), g["apply"]) < 1e-12
    for st in ("rgmres", "lgmres"):
        res = O.solve(sol_json(st, itmax=2000))
        assert res["flag"] == int(g[f"{st}_flag"])
        assert abs(res["iter"] - int(g[f"{st}_iter"])) <= max(1, 0.1 * int(g[f"{st}_iter"]))
        assert rel(res["x"], g[f"{st}_x"]) < 1e-6


LIVE = {
    "c1": lambda gen: gen.generate(gen.preset(1)),
    "bs3_faults": lambda gen: gen.grid(12, 10, 6, bs=3, fault_frac=0.02, layered=1, sigma=2.0, kz_kx=0.1),
    "channels": lambda gen: gen.grid(30, 20, 10, bs=2, seed=5, n_channels=3, channel_contrast=1e4, sigma=2.5,
                                     comp=1.0),
}


@pytest.mark.parametrize("name", list(LIVE))
@pytest.mark.parametrize("case", [dict(), dict(drs=1, e_ps=0.5), dict(seq=0, glo_rel=0.2),
                                  dict(glo_power=2, loc_power=2)])
def test_port_matches_reference_live(name, case):
    from deco_b200 import gen
    from oracle import port, ref
    if not ref.available():
        pytest.skip("reference library not built")
    s = LIVE[name](gen)
    prec = cpr_json(s.bs, **case)
    R = ref.Cpr({"prec": prec}, s.r, s.c, s.v, s.b)
    O = port.Cpr(prec, s.r, s.c, s.v, s.b)
    for a, b in zip(O.decoupled(), R.decoupled()):
        np.testing.assert_array_equal(a, b)  # bit-exact decoupling
    for a, b in zip(O.pressure(), R.pressure()):
        np.testing.assert_array_equal(a, b)
    for w in (0, 1):
        (OL, OU), (RL, RU) = O.fsai(w), R.fsai(w)
        for k in (0, 1):
            np.testing.assert_array_equal(OL[k], RL[k])
            np.testing.assert_array_equal(OU[k], RU[k])
        assert rel(OL[2], RL[2]) < 1e-13 and rel(OU[2], RU[2]) < 1e-13
    x = np.random.default_rng(3).standard_normal(s.n)
    assert rel(O.apply(x), R.apply(x)) < 1e-12
    if name == "c1" and not case:
        a = R.solve(sol_json())
        b = O.solve(sol_json())
        assert a["iter"] == b["iter"] and abs(a["res_rel"] - b["res_rel"]) < 1e-11


def test_reference_errors_are_reproduced_as_statuses():
    """The reference exits on a zero CPD determinant (CPR.hpp:643-646); the port returns a status."""
    from deco_b200 import gen
    from oracle import port
    s = gen.grid(4, 3, 2, bs=2, seed=1)
    v = s.v.copy()
    rows = np.repeat(np.arange(s.n), np.diff(s.r))
    v[(rows < 2) & (s.c < 2)] = 1.0
    with pytest.raises(RuntimeError):
        port.Cpr(cpr_json(2), s.r, s.c, v, s.b)
