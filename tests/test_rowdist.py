"""Row-partitioned CPR-GMRES (deco_b200/rowdist.py) on CPU: the halo plans, the
distributed CPR apply and right GMRES over two gloo ranks, against the same code
on one rank and against the oracle.  The local products run through scipy here
(the product path runs them through the library's SpMV on each rank's GPU); the
partitioning, halo exchange, all-reduces and recurrences are the code under test.

The operators are the oracle's CPR setup of the whole system (decoupled A, A_pp
and both FSAI factors), sliced by rows as every rank does with its own setup.
"""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


class ScipyProducts:
    """Local products of row slices on the CPU (scipy), the test's stand-in for
    LibraryProducts."""
    device = torch.device("cpu")

    def prepare(self, sl):
        import scipy.sparse as sp
        return sp.csr_matrix((sl.v, sl.c, sl.r), shape=(sl.rows, sl.ncols))

    def apply(self, M, xg, bs=1):
        y = M @ xg.numpy()
        return torch.from_numpy(np.ascontiguousarray(y[0::bs] if bs > 1 else y))


def _system():
    from deco_b200 import gen
    return gen.grid(12, 10, 8, bs=2, seed=21)


def _operators(s, prec):
    from oracle import port
    O = port.Cpr(prec, s.r, s.c, s.v, s.b)
    Ar, Ac, Av, Ab = O.decoupled()
    return O, (Ar, Ac, Av, Ab), O.pressure(), O.fsai(0), O.fsai(1)


def _run(rank, world, prec, sol):
    from deco_b200 import rowdist as rd
    s = _system()
    O, (Ar, Ac, Av, Ab), (Pr, Pc, Pv), ((Lr, Lc, Lv), (Ur, Uc, Uv)), ((lr, lc, lv), (ur, uc, uv)) = _operators(s, prec)
    bs = 2
    n, nc = s.n, s.n // bs
    displs = rd.split_rows(n, world, bs)
    r0, r1 = displs[rank], displs[rank + 1]
    c0, c1 = r0 // bs, r1 // bs
    sl = (rd.RowSlice.cut(Ar, Ac, Av, r0, r1, n), rd.RowSlice.cut(Lr, Lc, Lv, r0, r1, n),
          rd.RowSlice.cut(Ur, Uc, Uv, r0, r1, n), rd.RowSlice.cut(lr, lc, lv, c0, c1, nc),
          rd.RowSlice.cut(ur, uc, uv, c0, c1, nc))
    D = rd.DistCPR(ScipyProducts(), displs, rank, world, bs, 0, *sl)
    # the distributed CPR apply against the oracle's apply on the whole vector
    rv = np.random.default_rng(5).standard_normal(n)
    xd = D.apply(torch.from_numpy(rv[r0:r1].copy())).numpy()
    xo = O.apply(rv)[r0:r1]
    apply_err = float(np.linalg.norm(xd - xo) / np.linalg.norm(xo))
    x, it, res, flag = rd.rgmres(D, torch.from_numpy(Ab[r0:r1].copy()), int(sol["restart"]), float(sol["reltol"]),
                                 int(sol["itmax"]))
    halo = (D.hA.ghosts, D.hFL.ghosts, D.hFUt.ghosts)
    return x.numpy(), it, res, flag, apply_err, halo, displs


def _worker(rank, world, port, out, prec, sol):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        out[rank] = _run(rank, world, prec, sol)
    finally:
        dist.destroy_process_group()


def test_split_rows_follows_the_reference():
    from deco_b200 import rowdist as rd
    assert rd.split_rows(10, 3, 1) == [0, 3, 6, 10]
    assert rd.split_rows(960, 2, 2) == [0, 480, 960]
    assert rd.split_rows(30, 4, 3) == [0, 6, 12, 18, 30]  # floor(30/4) = 7 -> 6, the last rank takes the rest
    for n, w, bs in [(960, 3, 2), (1001, 4, 1), (999, 5, 3)]:
        d = rd.split_rows(n, w, bs)
        assert d[0] == 0 and d[-1] == n and all(b >= a for a, b in zip(d, d[1:]))
        assert all(x % bs == 0 for x in d[:-1])


def test_two_gloo_ranks_match_one_rank():
    """Two ranks: each rank's slice of the distributed CPR apply equals the oracle's
    apply within 1e-13; the distributed solve converges to 1e-8 in the one-rank
    solve's iteration count (within 10%; the all-reduced dots sum in another order)
    and to the same solution within 1e-9; the one-rank count is within 10% of the
    oracle's own rgmres (modified Gram-Schmidt there, CGS2 here)."""
    import torch.multiprocessing as mp
    from conftest import cpr_json, sol_json
    from oracle import port
    prec, sol = cpr_json(2), sol_json(restart=20)
    x1, it1, res1, flag1, aerr1, halo1, _ = _run(0, 1, prec, sol)
    assert flag1 == 0 and res1 < 1e-8 and aerr1 < 1e-13
    assert halo1 == (0, 0, 0)
    s = _system()
    ref_it = port.Cpr(prec, s.r, s.c, s.v, s.b).solve(sol)["iter"]
    assert abs(it1 - ref_it) <= max(1, 0.1 * ref_it), (it1, ref_it)
    world, port_ = 2, _free_port()
    mgr = mp.get_context("spawn").Manager()  # no fork of this multi-threaded process
    out = mgr.dict()
    mp.spawn(_worker, args=(world, port_, out, prec, sol), nprocs=world, join=True)
    xs = []
    for rank in range(world):
        x, it, res, flag, aerr, halo, displs = out[rank]
        assert flag == 0 and res < 1e-8, (rank, res)
        assert aerr < 1e-13, (rank, aerr)
        assert abs(it - it1) <= max(1, 0.1 * it1), (it, it1)
        assert halo[0] > 0, "the rank's rows must read ghost columns"
        xs.append(x)
    # the ranks ran the same recurrences: the same count everywhere
    assert out[0][1] == out[1][1]
    xd = np.concatenate(xs)
    assert np.linalg.norm(xd - x1) / np.linalg.norm(x1) < 1e-9
    # the lower block's FL rows read nothing from above; its FU^T rows do
    assert out[0][5][1] == 0 and out[0][5][2] > 0
    assert out[1][5][1] > 0 and out[1][5][2] == 0
