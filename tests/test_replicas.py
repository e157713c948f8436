"""N > 1 path on CPU: two gloo ranks, each solving its own seeded system with the
CPU oracle, aggregated the way bench.py aggregates GPU replicas."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from conftest import cpr_json, sol_json
        from deco_b200 import gen, replicas
        from oracle import port as oport
        mine = list(replicas.shard(5, rank, world))
        iters = 0
        worst = 0.0
        for k in mine:
            s = gen.grid(6, 5, 3, bs=2, seed=100 + k)
            O = oport.Cpr(cpr_json(2), s.r, s.c, s.v, s.b)
            res = O.solve(sol_json(itmax=500))
            assert res["flag"] == 0
            iters += res["iter"]
            worst = max(worst, res["res_rel"])
        out[rank] = (mine, replicas.max_over_ranks(float(len(mine))), replicas.sum_over_ranks(iters),
                     replicas.max_over_ranks(worst))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_share_independent_systems():
    import torch.multiprocessing as mp
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()  # no fork of this multi-threaded process
    out = mgr.dict()
    mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
    (m0, mx0, it0, w0), (m1, mx1, it1, w1) = out[0], out[1]
    assert sorted(m0 + m1) == list(range(5)) and not set(m0) & set(m1)
    assert mx0 == mx1 == 3.0  # max over ranks seen identically everywhere
    assert it0 == it1 > 0 and w0 == w1 < 1e-8


def test_shard_covers_everything_once():
    from deco_b200 import replicas
    for n in (0, 1, 7, 64):
        for world in (1, 2, 3, 8):
            got = [i for r in range(world) for i in replicas.shard(n, r, world)]
            assert got == list(range(n))
    with pytest.raises(ValueError):
        replicas.shard(4, 2, 2)


def _batch_worker(rank, world, port, out):
    """One rank of the batched bench's split on CPU: the systems replicas.deal gives this
    rank, cut from the full batch by gen.batch_subset, solved with the oracle; each
    system of the rank's block-diagonal share must be exactly that system of the batch."""
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import numpy as np
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from conftest import cpr_json, sol_json
        from deco_b200 import gen, replicas
        from oracle import port as oport
        nsys, K = 5, 2
        r, c, v, ro, B, shapes = gen.batch(nsys, 77, 60, 300, 2, K)
        mine = replicas.deal(nsys, rank, world)
        r2, c2, v2, ro2, B2 = gen.batch_subset(r, c, v, ro, B, K, mine)
        Bm, B2m = B.reshape(-1, K), B2.reshape(-1, K)
        worst, iters = 0.0, 0
        for t, q in enumerate(mine):
            # the share's block t is system q of the full batch, bit for bit
            a, e, a2, e2 = int(ro[q]), int(ro[q + 1]), int(ro2[t]), int(ro2[t + 1])
            assert e - a == e2 - a2
            np.testing.assert_array_equal(np.diff(r[a:e + 1]), np.diff(r2[a2:e2 + 1]))
            np.testing.assert_array_equal(c[r[a]:r[e]] - a, c2[r2[a2]:r2[e2]] - a2)
            np.testing.assert_array_equal(v[r[a]:r[e]], v2[r2[a2]:r2[e2]])
            np.testing.assert_array_equal(Bm[a:e], B2m[a2:e2])
        # the share solved as one block-diagonal system, one right-hand side per solve
        for k in range(K):
            O = oport.Cpr(cpr_json(2), r2, c2, v2, np.ascontiguousarray(B2m[:, k]))
            res = O.solve(sol_json(itmax=2000))
            assert res["flag"] == 0
            worst = max(worst, res["res_rel"])
            iters += res["iter"]
        out[rank] = (mine, replicas.sum_over_ranks(len(mine)), replicas.max_over_ranks(worst),
                     replicas.sum_over_ranks(iters))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_deal_the_batch():
    """The split bench.py's batched workload uses under torchrun (replicas.deal +
    gen.batch_subset), on two gloo ranks: every system lands on exactly one rank, each
    share holds those systems unchanged, and each share solves to 1e-8."""
    import torch.multiprocessing as mp
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()  # no fork of this multi-threaded process
    out = mgr.dict()
    mp.spawn(_batch_worker, args=(world, port, out), nprocs=world, join=True)
    (m0, n0, w0, i0), (m1, n1, w1, i1) = out[0], out[1]
    assert sorted(m0 + m1) == list(range(5)) and not set(m0) & set(m1)
    assert m0 == [0, 2, 4] and m1 == [1, 3]
    assert n0 == n1 == 5.0 and w0 == w1 < 1e-8 and i0 == i1 > 0


def test_deal_covers_everything_once():
    from deco_b200 import replicas
    for n in (0, 1, 7, 64):
        for world in (1, 2, 3, 8):
            got = sorted(i for r in range(world) for i in replicas.deal(n, r, world))
            assert got == list(range(n))
    with pytest.raises(ValueError):
        replicas.deal(4, 2, 2)
