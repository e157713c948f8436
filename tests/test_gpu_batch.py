"""Batched solve: many block-diagonal systems x several right-hand sides in one
lockstep CPR-GMRES, against solving each (system, column) pair on its own.

Bars: every instance converges (flag 0, decoupled true relative residual < 1e-8);
its iteration count is the single-system count within 2 (the same algorithm, with
the Arnoldi dots reduced in another order); its solution matches the single solve
within 1e-6 relative; the graph-replayed and the directly launched cycles give
bit-identical results.
"""
import os

import numpy as np
import pytest

from conftest import cpr_json, rel, sol_json
from deco_b200 import gen

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def d():
    import deco_b200
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    deco_b200.default_context()
    return deco_b200


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def subsystem(r, c, v, ro, q):
    a, e = r[ro[q]], r[ro[q + 1]]
    return (r[ro[q]:ro[q + 1] + 1] - a).astype(np.int32), (c[a:e] - ro[q]).astype(np.int32), v[a:e].copy()


@pytest.mark.parametrize("nrhs,restart", [(1, 50), (4, 50), (8, 50), (4, 5)])
def test_batch_matches_single_solves(d, nrhs, restart):
    """restart 5 makes every instance run several restart cycles."""
    r, c, v, ro, B, _ = gen.batch(5, seed=3, cells_lo=60, cells_hi=600, nrhs=nrhs)
    n = int(ro[-1])
    prec, sol = cpr_json(2), sol_json(restart=restart)
    A = d.CSR(n, n, r, c, v)
    Bt = d.Batch(prec, A, ro, nrhs)
    X = Bt.solve(sol, cuda(B)).cpu().numpy().reshape(n, nrhs)
    assert (Bt.flags == 0).all() and (Bt.res_rel < 1e-8).all()
    assert Bt.result["converged"] == 5 * nrhs
    Bm = B.reshape(n, nrhs)
    for q in range(5):
        rq, cq, vq = subsystem(r, c, v, ro, q)
        nq = len(rq) - 1
        for k in range(nrhs):
            A1 = d.CSR(nq, nq, rq, cq, vq)
            b1 = cuda(Bm[ro[q]:ro[q + 1], k])
            P1 = d.CPR(prec, A1, b1)
            S1 = d.SOL(sol, A1, P1, b1)
            assert abs(int(Bt.iters[q, k]) - S1.iter) <= 2, (q, k, Bt.iters[q, k], S1.iter)
            assert rel(X[ro[q]:ro[q + 1], k], S1.x.cpu().numpy()) < 1e-6


def test_batch_launch_modes_agree(d):
    """One graph launch with the device-side cycle loop (default), the cycle graph
    relaunched by the host, and direct launches: bit-identical results; restart 10
    makes the loop run several cycles."""
    r, c, v, ro, B, _ = gen.batch(4, seed=5, cells_lo=100, cells_hi=800, nrhs=4)
    n = int(ro[-1])
    out = []
    for mode in ("2", "1", "0"):
        os.environ["DECO_BATCH_GRAPH"] = mode
        try:
            Bt = d.Batch(cpr_json(2), d.CSR(n, n, r, c, v), ro, 4)
            X = Bt.solve(sol_json(restart=10), cuda(B)).cpu().numpy()
            out.append((X, Bt.iters.copy(), Bt.result["graph"], Bt.result["cycles"]))
            assert (Bt.flags == 0).all()
        finally:
            os.environ.pop("DECO_BATCH_GRAPH", None)
    assert [o[2] for o in out] == [2, 1, 0]
    assert out[0][3] == out[1][3] == out[2][3] > 1
    for o in out[1:]:
        np.testing.assert_array_equal(out[0][0], o[0])
        np.testing.assert_array_equal(out[0][1], o[1])


def test_batch_mixed_precision(d):
    """float32 preconditioner and basis with float64 refinement: every instance
    matches the single-system mixed solve (the float32 inner estimate can stop a
    cycle early and cost one more refinement cycle, as it does there)."""
    r, c, v, ro, B, _ = gen.batch(6, seed=7, cells_lo=200, cells_hi=2000, nrhs=8)
    n = int(ro[-1])
    prec, sol = cpr_json(2), sol_json()
    A = d.CSR(n, n, r, c, v)
    Bt = d.Batch(prec, A, ro, 8, precision=32)
    X = Bt.solve(sol, cuda(B)).cpu().numpy().reshape(n, 8)
    assert (Bt.flags == 0).all() and (Bt.res_rel < 1e-8).all()
    Bm = B.reshape(n, 8)
    for q in (0, 3, 5):
        rq, cq, vq = subsystem(r, c, v, ro, q)
        nq = len(rq) - 1
        for k in (0, 7):
            A1 = d.CSR(nq, nq, rq, cq, vq)
            b1 = cuda(Bm[ro[q]:ro[q + 1], k])
            P1 = d.CPR(prec, A1, b1, 32)
            S1 = d.SOL(sol, A1, P1, b1, precision=32)
            assert abs(int(Bt.iters[q, k]) - S1.iter) <= 2, (q, k, Bt.iters[q, k], S1.iter)
            assert rel(X[ro[q]:ro[q + 1], k], S1.x.cpu().numpy()) < 1e-6
    # and the float64 batch solution within the tolerance the solves reach
    X64 = d.Batch(prec, d.CSR(n, n, r, c, v), ro, 8).solve(sol, cuda(B)).cpu().numpy().reshape(n, 8)
    assert rel(X, X64) < 1e-6
    assert len(Bt.widths) == 6 and (Bt.widths >= 1).all()


def test_batch_errors(d):
    r, c, v, ro, B, _ = gen.batch(3, seed=9, cells_lo=60, cells_hi=200, nrhs=4)
    n = int(ro[-1])
    with pytest.raises(d.DecoError) as e:
        d.Batch(cpr_json(2), d.CSR(n, n, r, c, v), ro, 3)
    assert e.value.code == -6
    bad = ro.copy()
    bad[1] += 1  # not on a cell boundary
    with pytest.raises(d.DecoError) as e:
        d.Batch(cpr_json(2), d.CSR(n, n, r, c, v), bad, 4)
    assert e.value.code == -1
    with pytest.raises(d.DecoError) as e:
        d.Batch(cpr_json(2, seq=1), d.CSR(n, n, r, c, v), ro, 4)
    assert e.value.code == -6
