"""Multi-GPU batch partition: the host logic of the N > 1 path (bench.py under
torchrun) on CPU -- the LPT assignment and a world-size-2 gloo run in which each
rank factors its shard of a batch (with the CPU oracle standing in for its GPU)
and the ranks check, through collectives, that the shards cover the batch once
and every system is solved."""
import os
import socket

import numpy as np

from mfdag import problems as P
from mfdag import sharding


def test_lpt_balance_and_determinism():
    rng = np.random.default_rng(0)
    costs = [int(c) for c in rng.integers(1, 10_000, size=200)]
    for world in (1, 2, 3, 8):
        parts = sharding.shard_lpt(costs, world)
        assert sorted(i for p in parts for i in p) == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) <= sum(costs) / world + max(costs)       # LPT bound
        assert parts == sharding.shard_lpt(costs, world)             # deterministic


def test_system_cost_matches_reference_model():
    p = P.laplace2d(20)
    c = sharding.system_cost(p.n, p.col, p.row, p.order, max_zero=10)
    from oracle import oracle as O
    assert c == O.Oracle.analyze(p.n, p.col, p.row, nb=10, max_zero=10, order_perm=p.order).cost()


def _worker(rank, world, port, count):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    for q in (os.path.dirname(here), os.path.join(os.path.dirname(here), "multifrontal-dag_b200"), here):
        if q not in sys.path:
            sys.path.insert(0, q)
    from datetime import timedelta
    import torch
    import torch.distributed as dist
    from mfdag import problems as Pw
    from mfdag import sharding as Sw
    from oracle import oracle as O
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=120))
    try:
        systems = Pw.laplace2d_batch(count=count, seed=3, lo=8, hi=24)
        costs = [Sw.system_cost(q.n, q.col, q.row, q.order, 10) for q in systems]
        mine = Sw.shard_lpt(costs, world)[rank]
        worst = 0.0
        for i in mine:
            q = systems[i]
            o = O.Oracle.analyze(q.n, q.col, q.row, nb=10, max_zero=10, order_perm=q.order)
            assert o.factorize(q.val) == 0
            x = o.solve(q.rhs)
            worst = max(worst, Pw.backward_error(q.n, q.col, q.row, q.val, x, q.rhs))
        shards = [None] * world
        dist.all_gather_object(shards, mine)
        t = torch.tensor([worst, float(len(mine))], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        if rank == 0:
            flat = sorted(i for s in shards for i in s)
            assert flat == list(range(count)), "shards must cover the batch exactly once"
            assert t[0].item() <= 1e-12, t[0].item()
            assert t[1].item() < count                                  # both ranks got work
    finally:
        dist.destroy_process_group()


def test_batch_shards_world2_gloo():
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.spawn(_worker, args=(2, port, 24), nprocs=2, join=True)
