"""Pair sharding (CPU): the plan, and the sharded solve over two gloo ranks with a stand-in
solver, against the same solver run on all pairs in one process."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from robotfd_b200 import shard


def fake_solve(Ps, Qs, **kw):
    """A deterministic stand-in for distance_batch (no GPU): values from the pair's sizes."""
    out = []
    for P, Q in zip(Ps, Qs):
        n1, n2 = len(P), len(Q)
        out.append({"distance": n1 * 0.5 + n2 * 0.25 + kw.get("shift", 0.0), "dfd": float(n1),
                    "vefd": float(n2), "endpoint": 0.125, "lb": 1.0, "ub": 2.0,
                    "cells_nominal": n1 * n2, "cells_evaluated": n1 + n2, "cells_fp64": n1,
                    "cells_vefd": n2, "probes": (n1 + n2) % 7, "flags": 32})
    return out


def pairs(n=37, seed=0):
    rng = np.random.default_rng(seed)
    return [(np.zeros((int(a), 2)), np.zeros((int(b), 2))) for a, b in
            zip(rng.integers(2, 3000, size=n), rng.integers(2, 3000, size=n))]


def test_plan_covers_and_balances():
    rng = np.random.default_rng(1)
    costs = rng.lognormal(14, 1, size=4096)
    for world in (1, 2, 3, 8):
        shares = shard.plan(costs, world)
        flat = np.sort(np.concatenate(shares))
        assert np.array_equal(flat, np.arange(len(costs)))
        loads = [costs[s].sum() for s in shares]
        # longest-first greedy: within the largest single cost of the mean
        assert max(loads) - min(loads) <= costs.max() + 1e-6
        assert shard.plan(costs, world)[0].tolist() == shares[0].tolist()  # deterministic


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ps = pairs()
        got = shard.distance_batch_sharded(None, [p for p, _ in ps], [q_ for _, q_ in ps],
                                           solve=fake_solve, shift=1.5)
        q.put((rank, got))
    finally:
        dist.destroy_process_group()


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


@pytest.mark.timeout(120)
def test_sharded_solve_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=100) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    ps = pairs()
    want = fake_solve([p for p, _ in ps], [q_ for _, q_ in ps], shift=1.5)
    for rank in (0, 1):
        assert got[rank] == want
