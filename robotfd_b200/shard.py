"""Pair sharding over the GPUs of one node (one process per GPU, torch.distributed).

Pairs are independent: every rank computes the same plan (pairs sorted by cells, each given to
the least-loaded rank, ties to the lowest rank), solves its share with the batch engine on its
own GPU, and one all-gather of a fixed-width record per pair rebuilds the full result list,
in the callers' order, on every rank.  No collective touches the sweeps themselves.

    results = distance_batch_sharded(ctx, Ps, Qs, precise=True)   # under torchrun

The all-gather runs on the process group's device (CUDA tensors for NCCL, CPU for gloo).
"""
import numpy as np

# result record: the rfd_result fields, in this order, as float64 (counts are exact below 2^53)
FIELDS = ("distance", "dfd", "vefd", "endpoint", "lb", "ub", "cells_nominal", "cells_evaluated",
          "cells_fp64", "cells_vefd", "probes", "flags")
INT_FIELDS = {"cells_nominal", "cells_evaluated", "cells_fp64", "cells_vefd", "probes", "flags"}


def plan(costs, world):
    """Greedy longest-first assignment: a list of index arrays, one per rank (each ascending)."""
    costs = np.asarray(costs, dtype=np.float64)
    load = np.zeros(world)
    owner = np.empty(len(costs), dtype=np.int64)
    for k in np.argsort(-costs, kind="stable"):
        r = int(np.argmin(load))
        owner[k] = r
        load[r] += costs[k]
    return [np.nonzero(owner == r)[0] for r in range(world)]


def _pack(results):
    a = np.zeros((len(results), len(FIELDS)))
    for k, r in enumerate(results):
        a[k] = [float(r[f]) for f in FIELDS]
    return a


def _unpack(row):
    return {f: (int(v) if f in INT_FIELDS else float(v)) for f, v in zip(FIELDS, row)}


def distance_batch_sharded(ctx, Ps, Qs, group=None, solve=None, **kw):
    """Solves pair k of (Ps, Qs) on one rank of `group` and returns every pair's result on
    every rank.  `solve(Ps, Qs, **kw) -> list of result dicts` defaults to
    ctx.distance_batch."""
    import torch
    import torch.distributed as dist
    if len(Ps) != len(Qs):
        raise ValueError("Ps and Qs differ in length")
    solve = solve or ctx.distance_batch
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    costs = [len(p) * len(q) for p, q in zip(Ps, Qs)]
    shares = plan(costs, world)
    mine = shares[rank]
    res = solve([Ps[k] for k in mine], [Qs[k] for k in mine], **kw) if len(mine) else []
    width = max(len(s) for s in shares)
    backend = dist.get_backend(group)
    device = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    buf = torch.zeros((width, len(FIELDS)), dtype=torch.float64, device=device)
    if len(mine):
        buf[: len(mine)] = torch.from_numpy(_pack(res)).to(device)
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    out = [None] * len(Ps)
    for r, share in enumerate(shares):
        rows = parts[r].cpu().numpy()
        for i, k in enumerate(share):
            out[k] = _unpack(rows[i])
    return out
