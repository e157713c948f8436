"""GPU parity: every hot-path kernel through the C ABI against the CPU oracle
(the plain-C restatement, oracle/port.py) and the reference built from its own
sources (oracle/ref.py) on identical seeded inputs.

Bars (stated per test): integer/pattern data bit-exact; the CPR decoupling
bit-exact (it is written as the same sequence of IEEE operations); SpMV, FSAI
values and CPR apply within 1e-12 relative (2-norm) in float64; GMRES reaches the
same float64 true residual with iteration counts within 10%.
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


@pytest.fixture(scope="module")
def oracle():
    from oracle import port, ref
    return port, ref


SYSTEMS = {
    "c1": lambda: gen.generate(gen.preset(1)),
    "bs3_faults": lambda: gen.grid(12, 10, 6, bs=3, fault_frac=0.02, layered=1, sigma=2.0, kz_kx=0.1),
    "tiny": lambda: gen.grid(5, 4, 3, bs=2, seed=7),
}
_cache = {}


def system(name):
    if name not in _cache:
        _cache[name] = SYSTEMS[name]()
    return _cache[name]


def cuda(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    return t if dtype is None else t.to(dtype)


# ---------------------------------------------------------------- SpMV (a1)

@pytest.mark.parametrize("name", list(SYSTEMS))
@pytest.mark.parametrize("bs", [1, 2])
def test_spmv_matches_oracle(d, oracle, name, bs):
    port, ref = oracle
    s = system(name)
    A = d.CSR.from_system(s)
    x = np.random.default_rng(1).standard_normal(s.n)
    y = A.apply(cuda(x), bs=bs).cpu().numpy()
    assert rel(y, port.spmv(s.r, s.c, s.v, x, bs)) < 1e-12
    assert rel(y, ref.spmv(s.r, s.c, s.v, x, bs)) < 1e-12


@pytest.mark.parametrize("sw", [1, 2, 4, 8, 16, 32])
def test_spmv_every_subwarp_width(d, oracle, sw):
    port, _ = oracle
    s = system("c1")
    A = d.CSR.from_system(s)
    A.subwarp = sw
    x = np.random.default_rng(2).standard_normal(s.n)
    assert rel(A.apply(cuda(x)).cpu().numpy(), port.spmv(s.r, s.c, s.v, x)) < 1e-12


def test_spmv_f32(d, oracle):
    port, _ = oracle
    s = system("c1")
    A = d.CSR.from_system(s)
    x = np.random.default_rng(3).standard_normal(s.n)
    y = A.apply_f32(cuda(x, torch.float32)).cpu().numpy()
    assert rel(y, port.spmv(s.r, s.c, s.v, x.astype(np.float32).astype(np.float64))) < 1e-6


def test_residual(d, oracle):
    port, _ = oracle
    s = system("tiny")
    A = d.CSR.from_system(s)
    x = np.random.default_rng(4).standard_normal(s.n)
    r = A.residual(cuda(s.b), cuda(x)).cpu().numpy()
    assert rel(r, s.b - port.spmv(s.r, s.c, s.v, x)) < 1e-12


# ------------------------------------------------------------- FSAI (a2-a7)

@pytest.mark.parametrize("name", ["c1", "bs3_faults"])
@pytest.mark.parametrize("tols", [(0.0, 0.0), (0.0, 1e-16), (0.2, 1e-16)])
@pytest.mark.parametrize("power", [1, 2])
def test_fsai_matches_reference(d, oracle, name, tols, power):
    """power 2: the lower(A A) pattern (symbolic.tpp:149-172), local systems of larger order."""
    _, ref = oracle
    s = system(name)
    A = d.CSR.from_system(s)
    F = d.FSAI({"tol_rel": tols[0], "tol_abs": tols[1], "power": power}, A)
    (Lr, Lc, Lv), (Ur, Uc, Uv) = F.factors()
    R = ref.Fsai(s.r, s.c, s.v, tols[0], tols[1], power)
    (RLr, RLc, RLv), (RUr, RUc, RUv) = R.factors()
    # pattern: bit-exact
    for a, b in [(Lr, RLr), (Lc, RLc), (Ur, RUr), (Uc, RUc)]:
        np.testing.assert_array_equal(a, b)
    assert rel(Lv, RLv) < 1e-12 and rel(Uv, RUv) < 1e-12
    x = np.random.default_rng(5).standard_normal(s.n)
    assert rel(F.apply(cuda(x)).cpu().numpy(), R.apply(x)) < 1e-12


@pytest.mark.parametrize("name", ["c1", "bs3_faults"])
def test_fsai_apply_f32(d, oracle, name):
    """Float32 vectors through a precision-32 factor (the product the mixed CPR
    applies): within 1e-5 of the reference's float64 FSAI::apply on the same
    float32-rounded input; in place; a precision-64 factor is refused."""
    _, ref = oracle
    s = system(name)
    A = d.CSR.from_system(s)
    F = d.FSAI({"tol_rel": 0.0, "tol_abs": 0.0, "power": 1}, A, precision=32)
    x32 = np.random.default_rng(8).standard_normal(s.n).astype(np.float32)
    y = F.apply_f32(cuda(x32))
    assert y.dtype == torch.float32
    R = ref.Fsai(s.r, s.c, s.v, 0.0, 0.0, 1)
    assert rel(y.cpu().numpy().astype(np.float64), R.apply(x32.astype(np.float64))) < 1e-5
    xx = cuda(x32)
    F.apply_f32(xx, xx)
    assert torch.equal(xx, y)
    with pytest.raises(d.DecoError):
        d.FSAI({"tol_rel": 0.0, "tol_abs": 0.0, "power": 1}, A).apply_f32(cuda(x32))


def test_fsai_apply_in_place(d, oracle):
    s = system("tiny")
    A = d.CSR.from_system(s)
    F = d.FSAI({"tol_rel": 0.0, "tol_abs": 0.0, "power": 1}, A)
    x = cuda(np.random.default_rng(6).standard_normal(s.n))
    y = F.apply(x.clone())
    F.apply(x, x)  # FSAI::apply accepts x aliasing b (FSAI.hpp:40-47)
    assert torch.equal(x, y)


# ------------------------------------------------------------- CPR (a8-a14)

CPR_CASES = {
    "ge_seq3": dict(),
    "drs": dict(drs=1),
    "drs_eps": dict(drs=1, e_ps=0.5),
    "qimpes_seq0": dict(weights="quasiimpes", seq=0),
    "seq1_glo_filter": dict(seq=1, glo_rel=0.2),
    "tol_zero": dict(tol_zero=1e-14),
    "power2": dict(glo_power=2, loc_power=2),
    "no_weights": dict(weights="none"),
}


@pytest.mark.parametrize("name", ["c1", "bs3_faults"])
@pytest.mark.parametrize("case", list(CPR_CASES))
def test_cpr_setup_and_apply(d, oracle, name, case):
    port, ref = oracle
    s = system(name)
    prec = cpr_json(s.bs, **CPR_CASES[case])
    A = d.CSR.from_system(s)
    b = cuda(s.b)
    P = d.CPR(prec, A, b)
    O = port.Cpr(prec, s.r, s.c, s.v, s.b)
    # decoupled system: bit-identical to the oracle port (same IEEE operation sequence)
    r, c, v = A.download()
    Or, Oc, Ov, Ob = O.decoupled()
    np.testing.assert_array_equal(r, Or)
    np.testing.assert_array_equal(c, Oc)
    np.testing.assert_array_equal(v, Ov)
    np.testing.assert_array_equal(b.cpu().numpy(), Ob)
    pr, pc, pv = P.Ap.download()
    Opr, Opc, Opv = O.pressure()
    np.testing.assert_array_equal(pr, Opr)
    np.testing.assert_array_equal(pc, Opc)
    np.testing.assert_array_equal(pv, Opv)
    for which in (0, 1):
        (Lr, Lc, Lv), (Ur, Uc, Uv) = P.fsai(which).factors()
        (OLr, OLc, OLv), (OUr, OUc, OUv) = O.fsai(which)
        for a_, b_ in [(Lr, OLr), (Lc, OLc), (Ur, OUr), (Uc, OUc)]:
            np.testing.assert_array_equal(a_, b_)
        assert rel(Lv, OLv) < 1e-12 and rel(Uv, OUv) < 1e-12
    rv = np.random.default_rng(7).standard_normal(s.n)
    x = P.apply(cuda(rv)).cpu().numpy()
    assert rel(x, O.apply(rv)) < 1e-12
    # and the reference itself, on the same inputs
    R = ref.Cpr({"prec": prec}, s.r, s.c, s.v, s.b)
    Rr, Rc, Rv, Rb = R.decoupled()
    np.testing.assert_array_equal(c, Rc)
    if prec["weights"] == "quasiimpes":
        # the reference's quasi_IMPES weights come from LAPACK dgesv (CPR.hpp:364),
        # whose internal operation order is not reproducible: equal to rounding
        assert rel(v, Rv) < 1e-13
    else:
        np.testing.assert_array_equal(v, Rv)
    assert rel(x, R.apply(rv)) < 1e-12


@pytest.mark.parametrize("name", ["c1", "bs3_faults"])
@pytest.mark.parametrize("power", [1, 2])
def test_fsai_local_systems_bit_exact_vs_oracle(d, oracle, name, power):
    """The batched local solves follow the oracle's textbook LU with partial
    pivoting operation by operation, in every order class (8, 16 and 32 lanes per
    row, and one warp per row past order 32): both FSAI factors of a CPR setup
    equal the C restatement's bit for bit."""
    port, _ = oracle
    s = system(name)
    prec = cpr_json(s.bs, glo_power=power, loc_power=power)
    A = d.CSR.from_system(s)
    P = d.CPR(prec, A, cuda(s.b))
    O = port.Cpr(prec, s.r, s.c, s.v, s.b)
    orders = []
    for which in (0, 1):
        (Lr, Lc, Lv), (Ur, Uc, Uv) = P.fsai(which).factors()
        (OLr, OLc, OLv), (OUr, OUc, OUv) = O.fsai(which)
        np.testing.assert_array_equal(Lc, OLc)
        np.testing.assert_array_equal(Uc, OUc)
        np.testing.assert_array_equal(Lv, OLv)
        np.testing.assert_array_equal(Uv, OUv)
        orders.append(np.diff(Lr) - 1)
    k = np.concatenate(orders)
    print(f"{name} power {power}: local orders {k.min()}..{k.max()}, "
          f"rows per class (<=8, <=16, <=32, <=64): {[(k <= 8).sum(), ((k > 8) & (k <= 16)).sum(), ((k > 16) & (k <= 32)).sum(), (k > 32).sum()]}")


@pytest.mark.parametrize("name", ["c1", "bs3_faults"])
@pytest.mark.parametrize("weights", ["quasiimpes", "none"])
def test_cpr_pressure_id_1_matches_reference(d, oracle, name, weights):
    """pressure_id 1 (CPR.hpp:50): the quasi-IMPES weights solve B^T w = e_1 (CPR.hpp:336),
    A_pp is the in-block row/column 1 (local_matrix, CSR.hpp:338-420), and the apply
    restricts r at row s*bs+1 against the row-0 product and prolongs into row s*bs+1
    (CPR.hpp:241-256; fix_diag and IMPES keep their default row 0).  Against the reference
    build: pattern bit-exact, values equal (1e-13 for the LAPACK weights), apply 1e-12.
    With quasi-IMPES weights on these pressure-first systems the reference's own global
    FSAI factor holds non-finite values (its local systems turn singular once row 0 gets
    the weighted sum and row 1 the pressure role), so its apply is NaN there and only the
    setup is compared."""
    _, ref = oracle
    s = system(name)
    prec = cpr_json(s.bs, weights=weights)
    prec["pressure_id"] = "1"
    A = d.CSR.from_system(s)
    b = cuda(s.b)
    P = d.CPR(prec, A, b)
    R = ref.Cpr({"prec": prec}, s.r, s.c, s.v, s.b)
    r, c, v = A.download()
    Rr, Rc, Rv, Rb = R.decoupled()
    np.testing.assert_array_equal(r, Rr)
    np.testing.assert_array_equal(c, Rc)
    if weights == "none":
        np.testing.assert_array_equal(v, Rv)
        np.testing.assert_array_equal(b.cpu().numpy(), Rb)
    else:
        assert rel(v, Rv) < 1e-13 and rel(b.cpu().numpy(), Rb) < 1e-13
    pr, pc, pv = P.Ap.download()
    Rpr, Rpc, Rpv = R.pressure()
    np.testing.assert_array_equal(pr, Rpr)
    np.testing.assert_array_equal(pc, Rpc)
    assert rel(pv, Rpv) < 1e-13
    if weights == "none":
        rv = np.random.default_rng(17).standard_normal(s.n)
        assert rel(P.apply(cuda(rv)).cpu().numpy(), R.apply(rv)) < 1e-12


def test_cpr_pressure_id_quasiimpes_ge_refused(d):
    """quasi_IMPES_GE writes its 1x1 / 2x2 system from row 0 (CPR.hpp:402-409, 433-437): with
    pressure_id != 0 the reference indexes out of bounds, so the GPU path refuses it."""
    s = system("tiny")
    prec = cpr_json(2)
    prec["pressure_id"] = "1"
    with pytest.raises(d.DecoError) as e:
        d.CPR(prec, d.CSR.from_system(s), cuda(s.b))
    assert e.value.code == -6


def test_cpr_fix_diag_zero_saturation_diagonal(d, oracle):
    """fix_diag (CPR.hpp:753-840): zero saturation diagonals are replaced, then undone."""
    port, _ = oracle
    s = system("tiny")
    v = s.v.copy()
    rows = np.repeat(np.arange(s.n), np.diff(s.r))
    zero = (rows % 2 == 1) & (s.c == rows) & (rows < 12)
    v[zero] = 0.0
    prec = cpr_json(2, weights="none", cpd=0)
    A = d.CSR(s.n, s.n, s.r, s.c, v)
    P = d.CPR(prec, A, cuda(s.b))
    assert P.fixed_diagonals == int(zero.sum())
    O = port.Cpr(prec, s.r, s.c, v, s.b)
    np.testing.assert_array_equal(A.download()[2], O.decoupled()[2])


def test_cpr_errors(d):
    s = system("tiny")
    # block size that does not divide n
    A = d.CSR.from_system(s)
    with pytest.raises(d.DecoError):
        d.CPR(cpr_json(3), A, cuda(s.b))
    # singular diagonal block -> status, no exit
    v = s.v.copy()
    rows = np.repeat(np.arange(s.n), np.diff(s.r))
    cell0 = (rows < 2) & (s.c < 2)
    v[cell0] = 1.0
    A = d.CSR(s.n, s.n, s.r, s.c, v)
    with pytest.raises(d.DecoError) as e:
        d.CPR(cpr_json(2), A, cuda(s.b))
    assert e.value.code == -4
    # an unknown sequence is an argument error; hypre AMG stays on the CPU build
    with pytest.raises(d.DecoError) as e:
        d.CPR(cpr_json(2, seq=4), d.CSR.from_system(s), cuda(s.b))
    assert e.value.code == -1
    with pytest.raises(d.DecoError) as e:
        d.CPR(cpr_json(2, loc="hypre_AMG"), d.CSR.from_system(s), cuda(s.b))
    assert e.value.code == -6


# --------------------------------------------------------------- GMRES (a15-a17)

@pytest.mark.parametrize("name", ["c1", "bs3_faults"])
@pytest.mark.parametrize("stype", ["rgmres", "lgmres"])
def test_gmres_matches_reference(d, oracle, name, stype):
    port, ref = oracle
    s = system(name)
    prec = cpr_json(s.bs)
    sol = sol_json(stype)
    A = d.CSR.from_system(s)
    b = cuda(s.b)
    P = d.CPR(prec, A, b)
    S = d.SOL(sol, A, P, b)
    R = ref.Cpr({"prec": prec}, s.r, s.c, s.v, s.b)
    res = R.solve(sol)
    assert S.flag == 0 and res["flag"] == 0
    assert abs(S.iter - res["iter"]) <= max(1, 0.1 * res["iter"])
    # true residual of the GPU solution on the decoupled system, measured by the oracle
    Dr, Dc, Dv, Db = R.decoupled()
    x = S.x.cpu().numpy()
    if stype == "rgmres":
        true_rel = np.linalg.norm(Db - port.spmv(Dr, Dc, Dv, x)) / np.linalg.norm(Db)
        assert true_rel < 1e-8
        assert abs(S.res_rel - true_rel) <= 1e-3 * true_rel + 1e-14
    assert rel(x, res["x"]) < 1e-6


@pytest.mark.parametrize("stype", ["rgmres", "lgmres"])
@pytest.mark.parametrize("precision", [64, 32])
def test_gmres_restart_100_matches_reference(d, oracle, stype, precision):
    """restart 100, as every shipped parameter file sets it (param_norne.json:15): cycles
    longer than 64 columns (several block rows in the dot pass, the back substitution's
    triangle in opt-in shared memory).  Float64: iterations within 10% of the reference
    build's, x within 1e-6 of the reference's.  Mixed precision is iterative refinement:
    a float32 cycle cannot carry the true residual more than about six decades below the
    residual it started from, so a solve that the float64 path finishes inside one or two
    long cycles may need one more refinement cycle; the bar is the reference's count plus
    one restart cycle, x within 1e-5.  Right GMRES: float64 true residual below 1e-8."""
    port, ref = oracle
    s = system("c1")
    prec = cpr_json(s.bs)
    sol = sol_json(stype, restart=100)
    A = d.CSR.from_system(s)
    b = cuda(s.b)
    P = d.CPR(prec, A, b, precision=precision)
    S = d.SOL(sol, A, P, b, precision=precision)
    R = ref.Cpr({"prec": prec}, s.r, s.c, s.v, s.b)
    res = R.solve(sol)
    assert res["iter"] > 64, "the case must run cycles longer than 64 columns"
    assert S.flag == 0 and res["flag"] == 0
    if precision == 64:
        assert abs(S.iter - res["iter"]) <= max(1, 0.1 * res["iter"]), (S.iter, res["iter"])
    else:
        assert S.iter <= res["iter"] + 100, (S.iter, res["iter"])
    Dr, Dc, Dv, Db = R.decoupled()
    x = S.x.cpu().numpy()
    if stype == "rgmres":
        true_rel = np.linalg.norm(Db - port.spmv(Dr, Dc, Dv, x)) / np.linalg.norm(Db)
        assert true_rel < 1e-8
    err = rel(x, res["x"])
    print(f"restart 100 {stype} precision {precision}: {S.iter} iterations (reference {res['iter']}), "
          f"|x - x_ref| / |x_ref| = {err:.2e}")
    assert err < (1e-6 if precision == 64 else 1e-5)


@pytest.mark.parametrize("name", ["c1", "bs3_faults"])
def test_gmres_mixed_precision_reaches_fp64_residual(d, oracle, name):
    """precision 32: float32 CPR + float32 Krylov basis, float64 refinement.  The
    float64 true residual reaches 1e-8 and the error of the mixed solution against the
    reference's float64 solution is stated and below 1e-6 (relative, 2-norm).  The
    iteration count is within 10% of the reference's float64 count when the solve spans
    several restart cycles (c1: about 220 iterations; the 1.5M- and 8M-row systems are
    held to the same bar in test_gpu_configs.py).  A solve that the float64 path
    finishes inside one cycle (bs3_faults: 25 iterations) takes one more refinement
    cycle in mixed precision -- a float32 cycle does not carry the true residual from 1 to
    1e-8 -- so there the bar is the float64 count plus one restart cycle."""
    port, ref = oracle
    s = system(name)
    prec = cpr_json(s.bs)
    A = d.CSR.from_system(s)
    b = cuda(s.b)
    P = d.CPR(prec, A, b, precision=32)
    S = d.SOL(sol_json(), A, P, b, precision=32)
    R = ref.Cpr({"prec": prec}, s.r, s.c, s.v, s.b)
    res = R.solve(sol_json())
    ref_it = res["iter"]
    Dr, Dc, Dv, Db = R.decoupled()
    x = S.x.cpu().numpy()
    true_rel = np.linalg.norm(Db - port.spmv(Dr, Dc, Dv, x)) / np.linalg.norm(Db)
    err = rel(x, res["x"])
    print(f"mixed {name}: {S.iter} iterations (reference float64 {ref_it}), true residual {true_rel:.2e}, "
          f"|x_mixed - x_ref| / |x_ref| = {err:.2e}")
    assert S.flag == 0 and true_rel < 1e-8
    if ref_it > 50:
        assert abs(S.iter - ref_it) <= max(1, 0.1 * ref_it), (S.iter, ref_it)
    else:
        assert S.iter <= ref_it + 50, (S.iter, ref_it)
    assert err < 1e-6


ORIG_CASES = {
    "ge_cpd_bs2": ("c1", dict(), "rgmres", 64),
    "drs_bs2_mixed": ("c1", dict(drs=1, e_ps=0.05), "rgmres", 32),
    "qimpes_bs3_lgmres": ("bs3_faults", dict(weights="quasiimpes"), "lgmres", 64),
    "ge_bs3_no_cpd": ("bs3_faults", dict(cpd=0), "rgmres", 64),
}


@pytest.mark.parametrize("name", list(ORIG_CASES))
def test_gmres_reports_original_system_residual(d, oracle, name):
    """res_rel is on the decoupled system (as the reference reports it); res_rel_orig
    is ||b0 - A0 x|| / ||b0|| on the system before the CPR setup rewrote A and b,
    checked here against the original arrays on the CPU: within 1e-12 of ||b0||
    (forming b - A x at a residual of 1e-8 cancels eight digits, so both sides
    carry rounding of that size) plus 1e-6 relative."""
    port, _ = oracle
    sysname, kw, stype, precision = ORIG_CASES[name]
    s = system(sysname)
    A = d.CSR.from_system(s)
    b = cuda(s.b)
    P = d.CPR(cpr_json(s.bs, **kw), A, b, precision=precision)
    S = d.SOL(sol_json(type_=stype), A, P, b, precision=precision)
    assert S.flag == 0
    x = S.x.cpu().numpy()
    orig = np.linalg.norm(s.b - port.spmv(s.r, s.c, s.v, x)) / np.linalg.norm(s.b)
    assert abs(S.res_rel_orig - orig) <= 1e-6 * orig + 1e-12, (S.res_rel_orig, orig)
    # without a preconditioner the solve has no decoupling to undo: the two agree
    S0 = d.SOL(sol_json(itmax=5), A, None, b)
    assert abs(S0.res_rel_orig - S0.res_rel) <= 1e-12 * S0.res_rel


def test_gmres_no_preconditioner_and_x0(d):
    s = gen.grid(3, 3, 3, bs=2, seed=5)  # 54 rows: GMRES(60) is full GMRES
    A = d.CSR.from_system(s)
    b = cuda(s.b)
    S0 = d.SOL(sol_json(itmax=600, restart=60), A, None, b)
    assert S0.flag == 0 and S0.res_rel < 1e-8
    x0 = S0.x.clone()
    r0 = (A.residual(b, x0).norm() / b.norm()).item()
    assert r0 < 1e-8, (r0, S0.res_rel)
    # starting from a converged x0 the inner check fires at j = 0, yet the
    # reference still adds M^{-1}(g_0 v_0) to x (rgmres.tpp:106-112) and then
    # re-checks the true residual; with no preconditioner that perturbs x, so a
    # few more iterations follow.  Same behaviour here: converged again, flag 0.
    S1 = d.SOL(sol_json(itmax=600, restart=60), A, None, b, x=x0)
    assert S1.flag == 0 and S1.res_rel < 1e-8, (S1.iter, S1.res_rel, r0, S0.res_rel)
