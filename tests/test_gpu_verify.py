"""GPU results certified by the exact decision verifier (oracle/verify.c).

Every bracket [lb, ub] the engine returns -- single pairs, the batch with the learned bracket,
the FP32 filter and the coarse upper bound -- contains the exact Frechet distance, and the
GPU's decisions around the distance agree with the exact ones, both up to the rounding of
the reference's FP64 formulas.  That rounding is bounded per pair by the conditioning
slack below: the free-interval discriminant B^2 - 4AC loses about eps |x - a|^2 to
cancellation, so the radius at which an edge opens moves by about eps (|x - a| / r)^2
relatively, |x - a| at most the diameter of the two curves.

Curves with consecutive repeated points are excluded here: the reference's free interval of
a zero-length segment is [0, 1] at every radius (0 * inf = NaN, clamped by fmax / fmin), so
its decisions, which the engine reproduces, are not the exact ones for them
(test_repeated_points_follow_the_reference)."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

ULP = 2.0 ** -52


def pairs(built):
    out = [built.gen_pair(k % 2, 2 + k % 2, 60 + 45 * k, 90 + 30 * k, 10.0 ** (k % 4 - 1), 0.05,
                          31, k) for k in range(10)]
    rng = np.random.default_rng(9)
    for k in range(6):  # random walks, one of them against a one-point curve
        P = np.cumsum(rng.normal(size=(int(rng.integers(2, 300)), 2)), 0)
        Q = np.cumsum(rng.normal(size=(int(rng.integers(2, 300)), 2)), 0)
        out.append((P[:1] if k == 0 else P, Q))
    return out


def slack(P, Q, r):
    """Relative rounding slack of the FP64 decision at radius r (see the module docstring)."""
    both = np.concatenate([P, Q])
    diam = float(np.linalg.norm(both.max(0) - both.min(0)))
    return 8 * ULP * max(1.0, (diam / r) ** 2)


def certify(P, Q, res):
    lb, ub = res["lb"], res["ub"]
    assert lb <= res["distance"] <= ub
    assert oracle.verify_decision(P, Q, ub * (1 + slack(P, Q, ub))) == 1, res
    assert oracle.verify_decision(P, Q, lb * (1 - slack(P, Q, lb))) == -1, res


@pytest.mark.parametrize("precise", [True, False])
def test_single_pair_brackets_contain_exact_distance(ctx, built, precise):
    for P, Q in pairs(built):
        certify(P, Q, ctx.distance(P, Q, precise=precise))


def test_batch_brackets_contain_exact_distance(ctx, built):
    ps = pairs(built)
    Ps, Qs = [p for p, _ in ps], [q for _, q in ps]
    model = built.Model.pretrained(0)
    for kw in ({}, {"model": model}, {"precision": built.RFD_PREC_FP32_FILTER},
               {"coarse_ub": 4}, {"model": model, "coarse_ub": 4}):
        for (P, Q), res in zip(ps, ctx.distance_batch(Ps, Qs, precise=True, **kw)):
            certify(P, Q, res)


def flip(decide, lo, hi):
    """The smallest double in (lo, hi] at which decide() holds (decide(lo) false, hi true)."""
    a, b = lo, hi
    while True:
        m = 0.5 * (a + b)
        if m <= a or m >= b:
            return b
        if decide(m):
            b = m
        else:
            a = m


def test_gpu_decisions_near_the_threshold(ctx, built):
    """The exact threshold is pinned to the verifier's band [r_lo, r_hi]; outside that band,
    widened by the rounding slack, the GPU decides exactly."""
    tight = 0
    for P, Q in pairs(built)[:8]:
        fd = ctx.distance(P, Q, precise=True)["distance"]
        lo, hi = fd * 0.9, fd * 1.1
        r_hi = flip(lambda r: oracle.verify_decision(P, Q, r) == 1, lo, hi)
        r_lo = flip(lambda r: oracle.verify_decision(P, Q, r) != -1, lo, hi)
        w = slack(P, Q, fd)
        assert r_hi - r_lo <= w * fd
        tight += w <= 1e-12
        for k in (0, 1, 4, 64, 1 << 20):
            assert not ctx.decide(P, Q, r_lo * (1 - w) - k * ULP * fd)[0], k
            assert ctx.decide(P, Q, r_hi * (1 + w) + k * ULP * fd)[0], k
    assert tight >= 4


def test_repeated_points_follow_the_reference(ctx, built):
    """A repeated point: the peak of height 3 is missed by the reference's decision (its
    zero-length segment is free at every radius), and the engine reproduces that; without the
    repeat (the same curve, the same exact distance) both decide exactly.  The reference's own
    method (no VE-FD for pairs of at most 10000 cells) searches up from the endpoint bound and
    lands below 1; a VE-FD lower bound (precise mode) happens to hide it on this pair."""
    P = np.array([[0.0, 0], [1, 0], [1, 0], [2, 0]])
    Q = np.array([[0.0, 0], [1, 3], [2, 0]])
    for r in (1.0, 2.0, 2.9):
        assert oracle.verify_decision(P, Q, r) == -1
        assert oracle.decide(P, Q, r)[0] and ctx.decide(P, Q, r)[0]
        assert not ctx.decide(P[[0, 1, 3]], Q, r)[0]
    got = ctx.distance(P, Q)
    assert got["distance"] == oracle.distance(P, Q)["distance"] < 1.0
    certify(P, Q, ctx.distance(P[[0, 1, 3]], Q))


def without_repeats(P):
    keep = np.concatenate([[True], np.any(P[1:] != P[:-1], axis=1)])
    return P[keep]


def with_repeats(rng, P):
    """P with runs of repeated points (a trajectory's stationary periods)."""
    reps = rng.integers(1, 4, size=len(P)) * (rng.random(len(P)) < 0.2) + 1
    return np.repeat(P, reps, axis=0)


def test_drop_repeats_gives_the_exact_distance(ctx, built):
    P = np.array([[0.0, 0], [1, 0], [1, 0], [2, 0]])
    Q = np.array([[0.0, 0], [1, 3], [2, 0]])
    for precise in (False, True):
        a = ctx.distance(P, Q, precise=precise, drop_repeats=True)
        b = ctx.distance(P[[0, 1, 3]], Q, precise=precise)
        for key in ("distance", "lb", "ub", "dfd", "vefd", "endpoint", "probes", "cells_nominal"):
            assert a[key] == b[key], key
        certify(P, Q, a)
        assert abs(a["distance"] - 3.0) <= 1e-6


def test_drop_repeats_batch(ctx, built):
    rng = np.random.default_rng(4)
    ps = []
    for k in range(12):
        d = 2 + k % 2
        P = with_repeats(rng, np.cumsum(rng.normal(size=(int(rng.integers(2, 250)), d)), 0))
        Q = with_repeats(rng, np.cumsum(rng.normal(size=(int(rng.integers(2, 250)), d)), 0))
        ps.append((P, Q))
    ps.append((np.repeat([[1.0, 2.0]], 5, axis=0), ps[0][1]))  # a curve of one repeated point
    Ps, Qs = [p for p, _ in ps], [q for _, q in ps]
    for precise in (False, True):
        got = ctx.distance_batch(Ps, Qs, precise=precise, drop_repeats=True)
        want = ctx.distance_batch([without_repeats(p) for p in Ps],
                                  [without_repeats(q) for q in Qs], precise=precise)
        for (P, Q), a, b in zip(ps, got, want):
            for key in ("distance", "lb", "ub", "dfd", "vefd", "probes", "cells_nominal"):
                assert a[key] == b[key], key
            certify(P, Q, a)
        if not precise:
            # the reference's behaviour is kept by default: some pair comes out too small
            plain = ctx.distance_batch(Ps, Qs)
            assert any(a["distance"] < b["distance"] for a, b in zip(plain, got))


def test_drop_repeats_on_device_curves(ctx, built):
    """Device-memory curves are counted and compacted on the device: the results equal the
    host path's bit for bit, single pairs and batches, and a replayed CUDA graph reads the
    new call's curves."""
    import torch
    rng = np.random.default_rng(7)
    ps = []
    for k in range(10):
        d = 2 + k % 2
        P = with_repeats(rng, np.cumsum(rng.normal(size=(int(rng.integers(2, 700)), d)), 0))
        Q = with_repeats(rng, np.cumsum(rng.normal(size=(int(rng.integers(2, 700)), d)), 0))
        ps.append((P, Q))
    ps.append((np.repeat([[1.0, 2.0]], 5, axis=0), ps[0][1]))  # a curve of one repeated point
    ps.append((np.array([[0.5, 0.5]]), ps[2][1]))               # a one-point curve
    keys = ("distance", "lb", "ub", "dfd", "vefd", "endpoint", "probes", "cells_nominal", "flags")
    dev = [(torch.tensor(P, device="cuda"), torch.tensor(Q, device="cuda")) for P, Q in ps]
    for precise in (False, True):
        want = ctx.distance_batch([P for P, _ in ps], [Q for _, Q in ps], precise=precise,
                                  drop_repeats=True)
        for (P, Q), (a, b), w in zip(ps, dev, want):
            got = ctx.distance_device(a.data_ptr(), len(P), b.data_ptr(), len(Q), P.shape[1],
                                      precise=precise, drop_repeats=True)
            for key in keys:
                assert got[key] == w[key], (key, got[key], w[key])
        batch = ctx.distance_batch([(a.data_ptr(), len(P), P.shape[1]) for (P, _), (a, _) in zip(ps, dev)],
                                   [(b.data_ptr(), len(Q), Q.shape[1]) for (_, Q), (_, b) in zip(ps, dev)],
                                   precise=precise, drop_repeats=True, memory=built.RFD_MEM_DEVICE)
        for g, w in zip(batch, want):
            for key in keys:
                assert g[key] == w[key], (key, g[key], w[key])
    # graph replay: same kept sizes, other coordinates in other device buffers
    P, Q = ps[3]
    a, b = dev[3]
    kw = dict(precise=True, drop_repeats=True, memory=built.RFD_MEM_DEVICE, graph=True)
    first = ctx.distance_batch([(a.data_ptr(), len(P), P.shape[1])], [(b.data_ptr(), len(Q), Q.shape[1])], **kw)
    assert first[0]["distance"] == ctx.distance(P, Q, precise=True, drop_repeats=True)["distance"]
    P2, Q2 = P * 1.5 + 0.25, Q * 0.75
    a2, b2 = torch.tensor(P2, device="cuda"), torch.tensor(Q2, device="cuda")
    again = ctx.distance_batch([(a2.data_ptr(), len(P2), P2.shape[1])], [(b2.data_ptr(), len(Q2), Q2.shape[1])], **kw)
    assert again[0]["distance"] == ctx.distance(P2, Q2, precise=True, drop_repeats=True)["distance"]
