"""Multi-process plumbing on CPU: two gloo ranks split a batch of uneven
problems by cost, each "solves" its share (here: the oracle's SpMV of the
problem's right-hand side, on the CPU — the GPU path is exercised by the gpu
tests), and the gathered results equal a single-rank run; the job time is
the maximum over ranks."""
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

from psiboil_b200.dist import gather_results, max_over_ranks, my_share, shard_by_cost, sum_over_ranks


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _batch(oracle, n):
    return [oracle.Problem(oracle.KIND_BATCH, 3, index=i, n2d=n // 2, s2=(12, 40), s3=(6, 14))
            for i in range(n)]


def _work(oracle, P):
    y = oracle.spmv(P, P.b)
    return float(np.dot(y, P.b))


def _rank(rank, world, port, n, out):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "oracle")]
    import oracle_py
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        probs = _batch(oracle_py, n)
        costs = [P.N for P in probs]
        mine = my_share(costs, rank, world)
        local = {i: _work(oracle_py, probs[i]) for i in mine}
        res = gather_results(local)
        t = max_over_ranks(float(rank + 1))
        cells = sum_over_ranks(sum(costs[i] for i in mine))
        if rank == 0:
            out.put((res, t, cells, sum(costs)))
    finally:
        dist.destroy_process_group()


def test_shard_by_cost_partitions_and_balances():
    costs = [5, 1, 9, 3, 3, 7, 2, 8]
    for world in (1, 2, 3):
        owner = shard_by_cost(costs, world)
        assert sorted(set(owner)) == list(range(min(world, len(costs))))
        loads = [sum(c for c, o in zip(costs, owner) if o == r) for r in range(world)]
        assert max(loads) - min(loads) <= max(costs)
        shares = [my_share(costs, r, world) for r in range(world)]
        assert sorted(i for s in shares for i in s) == list(range(len(costs)))


def test_two_gloo_ranks_match_one(oracle):
    n = 10
    ref = {i: _work(oracle, P) for i, P in enumerate(_batch(oracle, n))}
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, n, q)) for r in range(2)]
    for p in procs:
        p.start()
    res, t, cells, total = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == ref
    assert t == 2.0
    assert cells == total
