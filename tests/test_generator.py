"""Synthetic systems: the named shapes, the CSR layout the reference's block
arithmetic needs, determinism."""
import numpy as np
import pytest

from deco_b200 import gen


@pytest.mark.parametrize("cfg,n,nnz", [(1, 64000, 870400), (5, 262144, 3604480), (3, 8000000, 111360000)])
def test_named_shapes(cfg, n, nnz):
    s = gen.generate(gen.preset(cfg))
    assert s.n == n and s.nnz == nnz


def test_config2_has_fault_connections():
    p = gen.preset(2)
    s = gen.generate(p)
    assert s.n == 1500000
    stencil_only = 9 * (7 * 500000 - 2 * (100 * 50 + 100 * 50 + 100 * 100))
    assert s.nnz > stencil_only  # 1% long-range pairs add dense 3x3 blocks


def layout_checks(s):
    r, c, v = s.r, s.c, s.v
    rows = np.repeat(np.arange(s.n), np.diff(r))
    # sorted, unique columns inside every row
    assert np.all((np.diff(c) > 0) | (np.diff(rows) != 0))
    # diagonal present in every row
    assert np.count_nonzero(c == rows) == s.n
    # every row of a cell has the same column pattern (precond/CPR.hpp:484-492)
    bs = s.bs
    lens = np.diff(r)
    assert np.all(lens.reshape(-1, bs) == lens.reshape(-1, bs)[:, :1])
    for cell in (0, s.n // bs // 2, s.n // bs - 1):
        base = c[r[cell * bs]:r[cell * bs + 1]]
        for p in range(1, bs):
            np.testing.assert_array_equal(c[r[cell * bs + p]:r[cell * bs + p + 1]], base)
    # dense bs x bs blocks: columns come in complete cell groups
    assert np.all(np.diff(r) % bs == 0)
    assert np.all(c.reshape(-1, bs) // bs == (c.reshape(-1, bs) // bs)[:, :1])
    assert np.all(np.isfinite(v)) and np.count_nonzero(v == 0.0) == 0


@pytest.mark.parametrize("kw", [dict(), dict(bs=3, fault_frac=0.05, layered=1), dict(n_channels=3, channel_contrast=1e4)])
def test_layout(kw):
    layout_checks(gen.grid(9, 7, 5, seed=3, **kw))


def test_structurally_symmetric_pattern():
    s = gen.grid(8, 6, 4, bs=3, seed=9, fault_frac=0.05)
    rows = np.repeat(np.arange(s.n), np.diff(s.r))
    a = set(zip(rows.tolist(), s.c.tolist()))
    assert all((j, i) in a for (i, j) in a)


def test_deterministic_and_seeded():
    a = gen.grid(10, 8, 6, seed=21)
    b = gen.grid(10, 8, 6, seed=21)
    c = gen.grid(10, 8, 6, seed=22)
    np.testing.assert_array_equal(a.v, b.v)
    np.testing.assert_array_equal(a.b, b.b)
    assert not np.array_equal(a.v, c.v)


def test_rhs_uniform():
    s = gen.generate(gen.preset(1))
    assert s.b.min() >= 0.0 and s.b.max() < 1.0 and abs(s.b.mean() - 0.5) < 0.01


def test_invalid_parameters_are_rejected():
    p = gen.preset(1)
    p.bs = 4
    with pytest.raises(ValueError):
        gen.generate(p)


def test_independent_of_thread_count():
    """Every draw is a counter-based hash and every reduction sums fixed chunks in
    order, so the system is the same for any OpenMP thread count."""
    import hashlib
    import os
    import subprocess
    import sys
    code = ("import sys, hashlib; sys.path.insert(0, %r); from deco_b200 import gen; "
            "s = gen.generate(gen.preset(5)); print(hashlib.md5(s.v.tobytes() + s.b.tobytes()).hexdigest())"
            % os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    digests = set()
    for t in ("1", "3", "8"):
        env = dict(os.environ, OMP_NUM_THREADS=t)
        out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, check=True)
        digests.add(out.stdout.strip())
    assert len(digests) == 1


def test_fill_from_logk_matches_seeded_field():
    p = gen.preset(1)
    p.nx, p.ny, p.nz = 7, 6, 4
    s = gen.generate(p, with_logk=True)
    t = gen.generate_from_logk(p, s.logk)
    np.testing.assert_array_equal(s.v, t.v)
    np.testing.assert_array_equal(s.c, t.c)
    np.testing.assert_array_equal(s.b, t.b)


@pytest.mark.parametrize("bs,kw", [(2, {}), (3, dict(fault_frac=0.05, layered=1))])
def test_grad_logk_matches_finite_differences(bs, kw):
    """L = <W, A(ln k)> for a fixed random W: the chain rule through the harmonic
    transmissibilities against central differences in every cell."""
    p = gen.preset(1)
    p.nx, p.ny, p.nz, p.bs = 5, 4, 3, bs
    for k, val in kw.items():
        setattr(p, k, val)
    s = gen.generate(p, with_logk=True)
    W = np.random.default_rng(0).standard_normal(s.nnz)
    g = gen.grad_logk(p, s.logk, W)
    g_seeded = gen.grad_logk(p, None, W)
    np.testing.assert_array_equal(g, g_seeded)
    h = 1e-4  # entries reach 1e5: smaller steps lose the difference to round-off
    fd = np.empty_like(g)
    for i in range(s.logk.size):
        lp = s.logk.copy(); lp[i] += h
        lm = s.logk.copy(); lm[i] -= h
        fd[i] = W @ (gen.generate_from_logk(p, lp).v - gen.generate_from_logk(p, lm).v) / (2 * h)
    np.testing.assert_allclose(g, fd, rtol=1e-6, atol=1e-8 * np.abs(fd).max())


def test_batch_blocks_and_subset():
    r, c, v, ro, B, shapes = gen.batch(5, seed=3, cells_lo=60, cells_hi=600, nrhs=4)
    assert len(ro) == 6 and ro[-1] == len(r) - 1 and len(B) == ro[-1] * 4
    rows = np.repeat(np.arange(ro[-1]), np.diff(r))
    sys_of = np.searchsorted(ro, rows, side="right") - 1
    assert (np.searchsorted(ro, c, side="right") - 1 == sys_of).all()  # block-diagonal
    cells = np.diff(ro) // 2
    assert (cells >= 2).all()
    r2, c2, v2, ro2, B2 = gen.batch_subset(r, c, v, ro, B, 4, [1, 3])
    for k, q in enumerate([1, 3]):
        a, e = ro[q], ro[q + 1]
        a2, e2 = ro2[k], ro2[k + 1]
        np.testing.assert_array_equal(r2[a2:e2 + 1] - r2[a2], r[a:e + 1] - r[a])
        np.testing.assert_array_equal(c2[r2[a2]:r2[e2]] - a2, c[r[a]:r[e]] - a)
        np.testing.assert_array_equal(v2[r2[a2]:r2[e2]], v[r[a]:r[e]])
        np.testing.assert_array_equal(B2.reshape(-1, 4)[a2:e2], B.reshape(-1, 4)[a:e])
