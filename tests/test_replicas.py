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
    mgr = mp.Manager()
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
