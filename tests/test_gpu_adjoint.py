"""GPU adjoint: transpose, right-hand-side decoupling replay, the on-pattern
gradient kernel, the adjoint solve, and the differentiable solve on the
64x64x32 two-phase workload with A assembled from a seeded log-permeability
field.

Bars: transpose, decoupling replay and gradient kernel bit-exact; dL/d ln k from
the GPU (float64 and mixed precision) within 1e-6 relative (2-norm) of the float64
CPU reference gradient (the reference's own CPR-GMRES on A and on A^T, at the
same 1e-10 tolerance); central finite differences of GPU forward solves on 50
random cells within 2e-3 relative (+1e-6 of the largest gradient).
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


PRECS = {
    "ge_cpd": dict(bs=2),
    "drs_eps": dict(bs=2, drs=1, e_ps=0.05),
    "qimpes_bs3": dict(bs=3, weights="quasiimpes"),
    "ge_bs3_drs": dict(bs=3, drs=1),
    "none_nocpd": dict(bs=2, weights="none", cpd=0),
}


@pytest.mark.parametrize("name", list(PRECS))
def test_decouple_rhs_replays_setup_bit_exact(d, name):
    kw = dict(PRECS[name])
    bs = kw.pop("bs")
    s = gen.grid(9, 7, 5, bs=bs, seed=5, fault_frac=0.02 if bs == 3 else 0.0)
    A = d.CSR.from_system(s)
    b = cuda(s.b)
    P = d.CPR(cpr_json(bs, **kw), A, b)
    b2 = P.decouple_rhs(cuda(s.b))
    np.testing.assert_array_equal(b2.cpu().numpy(), b.cpu().numpy())
    # any vector: decoupling is the block-diagonal left factor T, so T (A x) = (T A) x
    import scipy.sparse as sp
    x = np.random.default_rng(2).standard_normal(s.n)
    Ax = sp.csr_matrix((s.v, s.c, s.r), shape=(s.n, s.n)) @ x
    Dr, Dc, Dv = A.download()
    TAx = sp.csr_matrix((Dv, Dc, Dr), shape=(s.n, s.n)) @ x
    assert rel(P.decouple_rhs(cuda(Ax)).cpu().numpy(), TAx) < 1e-12


def test_decouple_rhs_replays_row_swap(d):
    """bs 3 cells whose second diagonal is zero get rows 1 and 2 swapped by
    fix_diag (precond/CPR.hpp:753-840); the replay swaps the same cells."""
    s = gen.grid(8, 6, 5, bs=3, seed=6)
    v = s.v.copy()
    rows = np.repeat(np.arange(s.n), np.diff(s.r))
    for cell in (3, 50, 101):
        i = 3 * cell + 1
        v[(rows == i) & (s.c == i)] = 0.0
    A = d.CSR(s.n, s.n, s.r, s.c, v)
    b = cuda(s.b)
    P = d.CPR(cpr_json(3), A, b)
    np.testing.assert_array_equal(P.decouple_rhs(cuda(s.b)).cpu().numpy(), b.cpu().numpy())


@pytest.mark.parametrize("shape", [(60, 60), (50, 37), (37, 50)])
def test_transpose_bit_exact(d, shape):
    import scipy.sparse as sp
    n, m = shape
    M = sp.random(n, m, density=0.1, random_state=n + m, format="csr")
    M.sort_indices()
    A = d.CSR(n, m, M.indptr.astype(np.int32), M.indices.astype(np.int32), M.data)
    T = A.transpose()
    assert (T.n, T.m, T.nz) == (m, n, M.nnz)
    r, c, v = T.download()
    Mt = M.T.tocsr()
    Mt.sort_indices()
    np.testing.assert_array_equal(r, Mt.indptr)
    np.testing.assert_array_equal(c, Mt.indices)
    np.testing.assert_array_equal(v, Mt.data)


def test_transpose_of_reservoir_matrix(d):
    from oracle import adjoint
    s = gen.grid(10, 8, 6, bs=3, seed=4, fault_frac=0.03)
    r, c, v = d.CSR.from_system(s).transpose().download()
    rt, ct, vt = adjoint.transpose(s.r, s.c, s.v, s.n)
    np.testing.assert_array_equal(r, rt)
    np.testing.assert_array_equal(c, ct)
    np.testing.assert_array_equal(v, vt)


@pytest.mark.parametrize("alpha", [-1.0, 0.5])
def test_grad_pattern_bit_exact(d, alpha):
    from oracle import adjoint
    s = gen.grid(11, 9, 7, bs=2, seed=8)
    rng = np.random.default_rng(1)
    lam, x = rng.standard_normal(s.n), rng.standard_normal(s.n)
    out = d.CSR.from_system(s).grad_pattern(cuda(lam), cuda(x), alpha).cpu().numpy()
    np.testing.assert_array_equal(out, adjoint.grad_pattern(s.r, s.c, lam, x, alpha))


@pytest.mark.parametrize("bs", [2, 3])
@pytest.mark.parametrize("precision", [64, 32])
def test_adjoint_solve_matches_reference(d, bs, precision):
    from oracle import adjoint, ref
    s = gen.grid(14, 12, 8, bs=bs, seed=3, fault_frac=0.01 if bs == 3 else 0.0)
    g = np.random.default_rng(4).random(s.n)
    prec, sol = cpr_json(bs), sol_json(reltol=1e-10)
    A = d.CSR.from_system(s)
    J = d.ADJ(prec, A, precision)
    lam = J.solve(sol, cuda(g)).cpu().numpy()
    assert J.flag == 0
    import scipy.sparse as sp
    At = sp.csr_matrix((s.v, s.c, s.r), shape=(s.n, s.n)).T
    assert np.linalg.norm(At @ lam - g) / np.linalg.norm(g) < 1e-8
    lam_ref = adjoint.adjoint(prec, sol, s.r, s.c, s.v, g, "ref" if ref.available() else "port")["x"]
    assert rel(lam, lam_ref) < 1e-7
    # A is unchanged by the adjoint setup; a second right-hand side reuses it
    np.testing.assert_array_equal(A.download()[2], s.v)
    lam2 = J.solve(sol, cuda(2.0 * g)).cpu().numpy()
    assert rel(lam2, 2.0 * lam) < 1e-8


# ------------------------------------------- the 64x64x32 log-permeability workload

OBS = 20
TOL = 1e-10


@pytest.fixture(scope="module")
def c5():
    p = gen.preset(5)
    s = gen.generate(p, with_logk=True)
    rng = np.random.default_rng(2024)
    obs = rng.choice(s.n // 2, OBS, replace=False)
    w = rng.random(OBS)
    return p, s, obs, w


@pytest.fixture(scope="module")
def c5_reference(c5):
    """float64 CPU reference: the reference's CPR-GMRES forward and on A^T."""
    from oracle import adjoint, ref
    p, s, obs, w = c5
    g = np.zeros(s.n)
    g[2 * obs] = w
    x, lam, gA, fwd, adj = adjoint.gradient(cpr_json(2), sol_json(reltol=TOL), s.r, s.c, s.v, s.b, g,
                                            "ref" if ref.available() else "port")
    assert fwd["flag"] == 0 and adj["flag"] == 0
    return dict(x=x, lam=lam, gA=gA, grad=gen.grad_logk(p, s.logk, gA))


def gpu_gradient(d, c5, precision):
    from deco_b200.adjoint import cpr_solve, last
    p, s, obs, w = c5
    values = cuda(s.v).requires_grad_(True)
    b = cuda(s.b).requires_grad_(True)
    x = cpr_solve(values, b, cuda(s.r), cuda(s.c), cpr_json(2), sol_json(reltol=TOL), precision)
    L = (cuda(w) * x[cuda(2 * obs)]).sum()
    L.backward()
    assert last.forward["flag"] == 0 and last.adjoint["flag"] == 0
    gA = values.grad.cpu().numpy()
    return x.detach().cpu().numpy(), b.grad.cpu().numpy(), gA, gen.grad_logk(p, s.logk, gA)


@pytest.mark.parametrize("precision", [64, 32])
def test_log_permeability_gradient_matches_cpu_reference(d, c5, c5_reference, precision):
    """The errors against the float64 CPU reference are stated for each result (x,
    lambda = dL/db, dL/dA, dL/d ln k) and bounded by 1e-6 relative."""
    x, gb, gA, grad = gpu_gradient(d, c5, precision)
    print(f"adjoint precision {precision}: |x - x_ref| {rel(x, c5_reference['x']):.2e}, "
          f"|lambda - lambda_ref| {rel(gb, c5_reference['lam']):.2e}, |dL/dA - ref| {rel(gA, c5_reference['gA']):.2e}, "
          f"|dL/dlnk - ref| {rel(grad, c5_reference['grad']):.2e} (relative, 2-norm)")
    assert rel(x, c5_reference["x"]) < 1e-6
    assert rel(gb, c5_reference["lam"]) < 1e-6       # dL/db = lambda
    assert rel(gA, c5_reference["gA"]) < 1e-6        # dL/dA on the pattern
    assert rel(grad, c5_reference["grad"]) < 1e-6    # chained to dL/d ln k


def test_log_permeability_gradient_matches_finite_differences(d, c5):
    import deco_b200
    p, s, obs, w = c5
    _, _, _, grad = gpu_gradient(d, c5, 64)
    prec, sol = cpr_json(2), sol_json(reltol=1e-11)

    def loss(lk):
        t = gen.generate_from_logk(p, lk)
        A = deco_b200.CSR.from_system(t)
        bb = cuda(t.b)
        P = deco_b200.CPR(prec, A, bb)
        S = deco_b200.SOL(sol, A, P, bb)
        assert S.flag == 0
        return float(w @ S.x.cpu().numpy()[2 * obs])

    h = 1e-2
    cells = np.random.default_rng(9).choice(s.logk.size, 50, replace=False)
    gmax = np.abs(grad).max()
    bad = []
    for i in cells:
        lp, lm = s.logk.copy(), s.logk.copy()
        lp[i] += h
        lm[i] -= h
        fd = (loss(lp) - loss(lm)) / (2 * h)
        if abs(fd - grad[i]) > 2e-3 * abs(grad[i]) + 1e-6 * gmax:
            bad.append((int(i), fd, grad[i]))
    assert not bad, bad
