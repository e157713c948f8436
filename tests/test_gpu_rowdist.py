"""The row-partitioned solve's product path on the GPU (one rank: the library's
SpMV on device row slices of a CPR setup made by the library), against the
single-GPU CPR apply and solve.  Several ranks need several GPUs; the
partitioning and exchanges are covered on CPU by test_rowdist.py."""
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


@pytest.mark.parametrize("bs", [2, 3])
def test_rowdist_one_rank_matches_single_gpu(d, bs):
    from deco_b200 import rowdist as rd
    s = gen.grid(16, 12, 8, bs=bs, seed=31, fault_frac=0.01 if bs == 3 else 0.0)
    prec, sol = cpr_json(bs), sol_json()
    # the distributed CPR apply against the library's own apply
    A = d.CSR.from_system(s)
    b = torch.from_numpy(s.b.copy()).cuda()
    P = d.CPR(prec, A, b)
    displs = rd.split_rows(s.n, 1, bs)
    D = rd.DistCPR(rd.LibraryProducts(), displs, 0, 1, bs, 0, *rd.slices_from_cpr(P, A, bs, displs, 0))
    rv = torch.from_numpy(np.random.default_rng(3).standard_normal(s.n)).cuda()
    assert rel(D.apply(rv.clone()).cpu().numpy(), P.apply(rv).cpu().numpy()) < 1e-12
    S = d.SOL(sol, A, P, b)
    x, it, res, flag, _ = rd.solve(prec, s, sol)
    assert flag == 0 and res < 1e-8
    assert abs(it - S.iter) <= max(1, 0.1 * S.iter), (it, S.iter)
    assert rel(x.cpu().numpy(), S.x.cpu().numpy()) < 1e-7
