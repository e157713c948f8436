"""The CPU reference gradient (oracle/adjoint.py) against dense linear algebra and
central finite differences, on systems small enough for dense solves."""
import numpy as np
import pytest
import scipy.sparse as sp

from deco_b200 import gen
from oracle import adjoint, ref

from conftest import cpr_json, rel, sol_json


def dense(s):
    return sp.csr_matrix((s.v, s.c, s.r), shape=(s.n, s.n)).toarray()


def test_transpose_matches_scipy():
    rng = np.random.default_rng(3)
    M = sp.random(37, 23, density=0.2, random_state=4, format="csr")
    M.sort_indices()
    rt, ct, vt = adjoint.transpose(M.indptr, M.indices, M.data, 23)
    T = M.T.tocsr()
    T.sort_indices()
    np.testing.assert_array_equal(rt, T.indptr)
    np.testing.assert_array_equal(ct, T.indices)
    np.testing.assert_array_equal(vt, T.data)
    del rng


@pytest.mark.parametrize("impl", ["port", "ref"])
@pytest.mark.parametrize("bs", [2, 3])
def test_gradient_matches_dense(impl, bs):
    if impl == "ref" and not ref.available():
        pytest.skip("reference not built")
    s = gen.grid(6, 5, 4, bs=bs, seed=11)
    rng = np.random.default_rng(1)
    g = np.zeros(s.n)
    g[bs * rng.choice(s.n // bs, 5, replace=False)] = rng.random(5)
    x, lam, gA, fwd, adj = adjoint.gradient(cpr_json(bs), sol_json(reltol=1e-13), s.r, s.c, s.v, s.b, g, impl)
    assert fwd["flag"] == 0 and adj["flag"] == 0
    D = dense(s)
    x_d = np.linalg.solve(D, s.b)
    lam_d = np.linalg.solve(D.T, g)
    assert rel(x, x_d) < 1e-10
    assert rel(lam, lam_d) < 1e-10
    rows = np.repeat(np.arange(s.n), np.diff(s.r))
    assert rel(gA, -lam_d[rows] * x_d[s.c]) < 1e-10


def test_chain_to_log_permeability_matches_finite_differences():
    """L = sum_k w_k p(cell_k): dL/d ln k = chain(dL/dA) + 0 (b does not depend on k),
    with dL/dA from the adjoint, against central differences of dense solves."""
    p = gen.preset(1)
    p.nx, p.ny, p.nz, p.bs = 6, 5, 3, 2
    s = gen.generate(p, with_logk=True)
    rng = np.random.default_rng(7)
    obs = rng.choice(s.n // 2, 6, replace=False)
    w = rng.random(6)
    g = np.zeros(s.n)
    g[2 * obs] = w
    _, _, gA, _, _ = adjoint.gradient(cpr_json(2), sol_json(reltol=1e-13), s.r, s.c, s.v, s.b, g, "port")
    grad = gen.grad_logk(p, s.logk, gA)

    def loss(lk):
        t = gen.generate_from_logk(p, lk)
        return w @ np.linalg.solve(dense(t), t.b)[2 * obs]

    h = 1e-4
    cells = rng.choice(s.logk.size, 12, replace=False)
    for i in cells:
        lp, lm = s.logk.copy(), s.logk.copy()
        lp[i] += h
        lm[i] -= h
        fd = (loss(lp) - loss(lm)) / (2 * h)
        assert abs(fd - grad[i]) <= 1e-5 * abs(grad[i]) + 1e-9 * np.abs(grad).max(), (i, fd, grad[i])
