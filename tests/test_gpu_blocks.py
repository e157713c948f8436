"""The cell-block (one index per bs x bs block) products against the CPU oracle.

Bars: float64 products within 1e-12 relative of the oracle's SpMV (core/alg.hpp:50-64)
for all rows and for the restricted product over row 0 of every cell; float32 values
within 1e-6; padding with explicit zeros leaves the product unchanged; CPR apply and
the solve through block copies keep the CPR parity bars.
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


SYSTEMS = {
    "c1_bs2": lambda: gen.generate(gen.preset(1)),
    "bs3_faults": lambda: gen.grid(12, 10, 6, bs=3, fault_frac=0.02, layered=1, sigma=2.0),
    "bs2_small": lambda: gen.grid(5, 4, 3, bs=2, seed=7),
}


def blocks_per_cell(r, c, bs):
    n = len(r) - 1
    cells = np.repeat(np.arange(n) // bs, np.diff(r))
    ncell = n // bs
    u = np.unique(cells.astype(np.int64) * (c.max() // bs + 1) + c // bs)
    return np.bincount(u // (c.max() // bs + 1), minlength=ncell)


def expected_slots(s, bs, nblk):
    ncell = s.n // bs
    if bs == 2:
        return 7 if 7 * ncell <= 1.25 * nblk else 0
    cnt = blocks_per_cell(s.r, s.c, bs)
    for w in (4, 7, 8):
        if (cnt > w).sum() <= ncell // 50 and w * ncell <= 1.25 * nblk:
            return w
    return 0


@pytest.mark.parametrize("name", list(SYSTEMS))
def test_block_products_match_oracle(d, name):
    from oracle import port
    s = SYSTEMS[name]()
    A = d.CSR.from_system(s)
    A.set_blocks(s.bs)
    bs, nblk = A.blocks
    assert bs == s.bs and nblk * bs * bs == s.nnz  # generated systems are dense cell blocks
    # 7-point cells carry up to 7 blocks: 7 padded slots when that pads at most 25 %;
    # 3x3 cells take the fewest of 4, 7, 8 slots that leave at most 2 % of the cells
    # to the overflow list within 25 % padding
    assert A.padded == expected_slots(s, bs, nblk)
    x = np.random.default_rng(0).standard_normal(s.n)
    assert rel(A.apply(cuda(x)).cpu().numpy(), port.spmv(s.r, s.c, s.v, x)) < 1e-12
    assert rel(A.apply(cuda(x), bs=s.bs).cpu().numpy(), port.spmv(s.r, s.c, s.v, x, s.bs)) < 1e-12
    y32 = A.apply_f32(cuda(x.astype(np.float32))).cpu().numpy()
    v32 = s.v.astype(np.float32).astype(np.float64)
    assert rel(y32, port.spmv(s.r, s.c, v32, x.astype(np.float32).astype(np.float64))) < 1e-6
    # a pointer not aligned for the pair loads takes the scalar path, same result
    xx = cuda(np.concatenate([[0.0], x]))
    assert rel(A.apply(xx[1:]).cpu().numpy(), port.spmv(s.r, s.c, s.v, x)) < 1e-12
    A.set_blocks(0)
    assert A.blocks == (0, 0)


def test_padded_copy_products(d):
    """The slot-padded 2x2 copy (products of matrices with at most 4 blocks per
    cell, as the FSAI factors of 7-point systems): a rectangular matrix with empty
    cells and 0-4 blocks per cell; full, row-0 and float32 products against the
    oracle; unused slots read a valid column with zero values."""
    from oracle import port
    rng = np.random.default_rng(9)
    ncell, mcell = 500, 300
    rows, cols = [], []
    for s_ in range(ncell):
        cs = np.sort(rng.choice(mcell, int(rng.integers(0, 5)), replace=False))
        for i in range(2):
            for c_ in cs:
                rows += [2 * s_ + i] * 2
                cols += [2 * c_, 2 * c_ + 1]
    rows, cols = np.array(rows), np.array(cols, dtype=np.int32)
    r = np.zeros(2 * ncell + 1, np.int32)
    np.cumsum(np.bincount(rows, minlength=2 * ncell), out=r[1:])
    v = rng.standard_normal(len(cols))
    A = d.CSR(2 * ncell, 2 * mcell, r, cols, v)
    A.set_blocks(2)
    assert A.blocks[0] == 2 and A.padded == 4
    x = rng.standard_normal(2 * mcell)
    assert rel(A.apply(cuda(x)).cpu().numpy(), port.spmv(r, cols, v, x)) < 1e-12
    assert rel(A.apply(cuda(x), bs=2).cpu().numpy(), port.spmv(r, cols, v, x, 2)) < 1e-12
    y32 = A.apply_f32(cuda(x.astype(np.float32))).cpu().numpy()
    assert rel(y32, port.spmv(r, cols, v.astype(np.float32).astype(np.float64),
                              x.astype(np.float32).astype(np.float64))) < 1e-6
    A.set_blocks(0)
    assert A.padded == 0


@pytest.mark.parametrize("precision", [64, 32])
def test_padded_3x3_copy_with_overflow(d, precision):
    """The slot-padded 3x3 copy: a rectangular matrix whose cells mostly carry
    3-4 blocks (1 % none) while 1 % carry 9-12, so 4 slots hold every cell but those, which
    keep 3 blocks in slots and the rest in the overflow list.  Full and row-0
    float64 products and the float32 product against the oracle."""
    from oracle import port
    rng = np.random.default_rng(31)
    ncell, mcell = 3000, 2000
    pick = rng.choice(ncell, ncell // 50, replace=False).tolist()
    wide, empty = set(pick[: ncell // 100]), set(pick[ncell // 100:])
    rows, cols = [], []
    for s_ in range(ncell):
        nb = int(rng.integers(9, 13)) if s_ in wide else (0 if s_ in empty else int(rng.integers(3, 5)))
        cs = np.sort(rng.choice(mcell, nb, replace=False))
        for i in range(3):
            for c_ in cs:
                rows += [3 * s_ + i] * 3
                cols += [3 * c_, 3 * c_ + 1, 3 * c_ + 2]
    rows, cols = np.array(rows), np.array(cols, dtype=np.int32)
    r = np.zeros(3 * ncell + 1, np.int32)
    np.cumsum(np.bincount(rows, minlength=3 * ncell), out=r[1:])
    v = rng.standard_normal(len(cols))
    A = d.CSR(3 * ncell, 3 * mcell, r, cols, v)
    A.set_blocks(3)
    assert A.blocks[0] == 3 and A.padded == 4
    x = rng.standard_normal(3 * mcell)
    if precision == 64:
        assert rel(A.apply(cuda(x)).cpu().numpy(), port.spmv(r, cols, v, x)) < 1e-12
        assert rel(A.apply(cuda(x), bs=3).cpu().numpy(), port.spmv(r, cols, v, x, 3)) < 1e-12
    else:
        y32 = A.apply_f32(cuda(x.astype(np.float32))).cpu().numpy()
        assert rel(y32, port.spmv(r, cols, v.astype(np.float32).astype(np.float64),
                                  x.astype(np.float32).astype(np.float64))) < 1e-6
    A.set_blocks(0)
    assert A.padded == 0


@pytest.mark.parametrize("precision", [64, 32])
def test_padded_copies_of_three_phase_cpr_with_faults(d, precision):
    """A three-phase system with fault connections: its global FSAI factors get the
    3x3 padded copy, and its pressure FSAI factors the scalar one with 4 slots, the
    rows lengthened by a fault (1.4 % of them) finishing from the overflow list.
    The CPR apply keeps the parity bar against the oracle and the solve its
    iteration count (mixed precision: a solve that float64 finishes inside one
    restart cycle takes one more refinement cycle, so there the bar is the count
    plus one cycle)."""
    from oracle import port
    s = SYSTEMS["bs3_faults"]()
    prec = cpr_json(3)
    A = d.CSR.from_system(s)
    b = cuda(s.b)
    P = d.CPR(prec, A, b, precision)
    assert P.fsai(0).padded[0] in (4, 7, 8) and P.fsai(1).padded == (4, 4)
    O = port.Cpr(prec, s.r, s.c, s.v, s.b)
    rvec = np.random.default_rng(6).standard_normal(s.n)
    tol = 1e-12 if precision == 64 else 1e-5
    assert rel(P.apply(cuda(rvec)).cpu().numpy(), O.apply(rvec)) < tol
    S = d.SOL(sol_json(), A, P, b, precision=precision)
    ref_it = O.solve(sol_json())["iter"]
    slack = max(2, 0.1 * ref_it) if precision == 64 else int(sol_json()["restart"])
    assert S.flag == 0 and abs(S.iter - ref_it) <= slack


def test_padding_with_zeros(d):
    """Entries missing from a cell block (a filtered pattern) are stored as zeros."""
    from oracle import port
    s = gen.grid(9, 8, 5, bs=2, seed=3)
    keep = np.ones(s.nnz, bool)
    rows = np.repeat(np.arange(s.n), np.diff(s.r))
    drop = (rows % 2 == 0) & (s.c % 2 == 1) & (s.c // 2 != rows // 2)  # p rows lose their s columns off the diagonal
    drop &= np.random.default_rng(1).random(s.nnz) < 0.3
    keep &= ~drop
    c, v = s.c[keep], s.v[keep]
    r = np.zeros(s.n + 1, np.int32)
    np.cumsum(np.bincount(rows[keep], minlength=s.n), out=r[1:])
    A = d.CSR(s.n, s.n, r, c, v)
    A.set_blocks(2)
    bs, nblk = A.blocks
    assert bs == 2 and nblk * 4 > len(c)
    x = np.random.default_rng(2).standard_normal(s.n)
    assert rel(A.apply(cuda(x)).cpu().numpy(), port.spmv(r, c, v, x)) < 1e-12


def test_too_much_padding_keeps_csr(d):
    """A scalar (diagonal-only) matrix would be 4x padded: no block copy is made."""
    n = 1000
    r = np.arange(n + 1, dtype=np.int32)
    c = np.arange(n, dtype=np.int32)
    A = d.CSR(n, n, r, c, np.ones(n))
    A.set_blocks(2)
    assert A.blocks == (0, 0)
    assert rel(A.apply(cuda(np.arange(n, dtype=np.float64))).cpu().numpy(), np.arange(n, dtype=np.float64)) == 0


@pytest.mark.parametrize("precision", [64, 32])
def test_cpr_builds_blocks_and_keeps_parity(d, precision):
    from oracle import port
    s = gen.generate(gen.preset(1))
    prec = cpr_json(2)
    A = d.CSR.from_system(s)
    b = cuda(s.b)
    P = d.CPR(prec, A, b, precision)
    assert A.blocks[0] == 2
    assert P.fsai(0).n == s.n
    # power-1 factors of a 7-point system: at most 4 blocks per cell (global FSAI)
    # and 4 entries per row (pressure FSAI) -> 4 padded slots
    assert P.fsai(0).padded == (4, 4)
    assert P.fsai(1).padded == (4, 4)
    O = port.Cpr(prec, s.r, s.c, s.v, s.b)
    rvec = np.random.default_rng(5).standard_normal(s.n)
    tol = 1e-12 if precision == 64 else 1e-5
    assert rel(P.apply(cuda(rvec)).cpu().numpy(), O.apply(rvec)) < tol
    S = d.SOL(sol_json(), A, P, b, precision=precision)
    ref_it = O.solve(sol_json())["iter"]
    assert S.flag == 0 and abs(S.iter - ref_it) <= max(2, 0.1 * ref_it)


@pytest.mark.parametrize("precision", [64, 32])
def test_product_plan_chosen_by_the_cpr_autotuner(d, precision):
    """A CPR setup times the products each of its matrices has a layout for (slot-padded
    copy, cell-block kernel, CSR kernel) and keeps the fastest; the chosen product of A
    is reported, and the CPR apply through it still matches the oracle."""
    from conftest import cpr_json
    from oracle import port
    s = gen.generate(gen.preset(1))
    A = d.CSR.from_system(s)
    b = torch.from_numpy(s.b.copy()).cuda()
    P = d.CPR(cpr_json(2), A, b, precision=precision)
    kind, lanes = A.product_plan(precision)
    assert kind in ("padded", "cells", "csr") and lanes >= 1
    if precision == 64:
        O = port.Cpr(cpr_json(2), s.r, s.c, s.v, s.b)
        rv = np.random.default_rng(9).standard_normal(s.n)
        x = P.apply(torch.from_numpy(rv).cuda()).cpu().numpy()
        xo = O.apply(rv)
        assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-12


@pytest.mark.parametrize("precision", [64, 32])
def test_slot_codes_give_bit_identical_solves(d, precision):
    """On a 7-point stencil the slots' column offsets take a handful of values, so the
    padded copies store 1-byte codes instead of 4-byte columns: the CPR setup and the
    solve must match a context that keeps 4-byte columns (DECO_SLOT_CODES=0) bit for bit."""
    import os
    from conftest import cpr_json, sol_json
    s = gen.grid(128, 100, 50, bs=2, seed=5)  # 640k cells: 7 slots x 640k, past the 2^22-slot coding threshold
    out = []
    for codes in ("1", "0"):
        os.environ["DECO_SLOT_CODES"] = codes
        try:
            ctx = d.Context(0)
        finally:
            os.environ.pop("DECO_SLOT_CODES", None)
        A = d.CSR.from_system(s, ctx)
        b = torch.from_numpy(s.b.copy()).cuda()
        P = d.CPR(cpr_json(2), A, b, precision=precision)
        S = d.SOL(sol_json(), A, P, b, precision=precision)
        ctx.sync()
        out.append((A.slot_codes, S.iter, S.x.cpu().numpy()))
    (bytes_on, noff_on), it_on, x_on = out[0]
    (bytes_off, _), it_off, x_off = out[1]
    assert bytes_on == 1 and 1 <= noff_on <= 256, out[0][0]
    assert bytes_off == 4
    assert it_on == it_off
    np.testing.assert_array_equal(x_on, x_off)
