"""Jacobi stages on the GPU against the reference build: apply_seq2 (its block
Jacobi first stage, CPR.hpp:202-233 with Jacobi.tpp:26-69), Jacobi as the global
(CPR<...,Jacobi,FSAI>) or local (CPR<...,FSAI,Jacobi>) preconditioner, point and
block forms.

Bars: CPR apply within 1e-12 relative of the reference (the block inverses come
from LAPACK dgetrf/dgetri there and from Gauss-Jordan here, equal to rounding);
GMRES iteration counts within 10% and the same float64 true residual.
"""
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


CASES = {
    "seq2_block": (2, dict(seq=2)),
    "seq2_point": (2, dict(seq=2, glo_bs=1)),
    "glo_jacobi_seq3": (2, dict(glo="Jacobi")),
    "glo_jacobi_seq1": (2, dict(glo="Jacobi", seq=1)),
    "loc_jacobi": (2, dict(loc="Jacobi")),
    "both_jacobi": (2, dict(glo="Jacobi", loc="Jacobi")),
    "bs3_seq2_no_cpd": (3, dict(seq=2, cpd=0, weights="quasiimpes")),
    "bs3_glo_jacobi_no_cpd": (3, dict(glo="Jacobi", cpd=0)),
}


def system(bs):
    if bs == 2:
        return gen.generate(gen.preset(1))
    return gen.grid(12, 10, 6, bs=3, fault_frac=0.02, layered=1, sigma=2.0)


@pytest.mark.parametrize("name", list(CASES))
def test_jacobi_stages_match_reference(d, name):
    from oracle import ref
    if not ref.available():
        pytest.skip("reference not built")
    bs, kw = CASES[name]
    s = system(bs)
    prec = cpr_json(bs, **kw)
    A = d.CSR.from_system(s)
    b = cuda(s.b)
    P = d.CPR(prec, A, b)
    R = ref.Cpr({"prec": prec}, s.r, s.c, s.v, s.b)
    Dr, Dc, Dv, Db = R.decoupled()
    if kw.get("weights") == "quasiimpes":  # LAPACK dgesv weights (CPR.hpp:364): equal to rounding
        assert rel(b.cpu().numpy(), Db) < 1e-13
    else:
        np.testing.assert_array_equal(b.cpu().numpy(), Db)
    rvec = np.random.default_rng(3).standard_normal(s.n)
    assert rel(P.apply(cuda(rvec)).cpu().numpy(), R.apply(rvec)) < 1e-12
    sol = sol_json(itmax=3000)
    S = d.SOL(sol, A, P, b)
    res = R.solve(sol)
    assert S.flag == 0 and res["flag"] == 0
    assert abs(S.iter - res["iter"]) <= max(2, 0.1 * res["iter"])
    x = S.x.cpu().numpy()
    import scipy.sparse as sp
    true_rel = np.linalg.norm(Db - sp.csr_matrix((Dv, Dc, Dr), shape=(s.n, s.n)) @ x) / np.linalg.norm(Db)
    assert true_rel < 1e-8


@pytest.mark.parametrize("name", ["seq2_block", "glo_jacobi_seq3"])
def test_jacobi_mixed_precision(d, name):
    bs, kw = CASES[name]
    s = system(bs)
    prec = cpr_json(bs, **kw)
    A = d.CSR.from_system(s)
    b = cuda(s.b)
    P = d.CPR(prec, A, b, precision=32)
    S = d.SOL(sol_json(itmax=3000), A, P, b, precision=32)
    assert S.flag == 0
    r = A.residual(b, S.x)
    assert (r.norm() / b.norm()).item() < 1e-8


def test_fsai_handle_of_a_jacobi_stage_is_an_error(d):
    s = system(2)
    A = d.CSR.from_system(s)
    P = d.CPR(cpr_json(2, glo="Jacobi"), A, cuda(s.b))
    with pytest.raises(d.DecoError):
        P.fsai(0)
    assert P.fsai(1).n == s.n // 2
