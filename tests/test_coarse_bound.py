"""The coarse upper bound's argument, on the CPU: the inflated DFD of the anchors (every k-th
point and the last; each anchor inflated by the radius of the block prefix after it and of
the block suffix before it, the blocks split at their middle index) is at least the DFD of the
full curves.  A restatement of coarse_prep_kernel + dfd_kernel<..., INFL=true> in numpy, checked
against the oracle's exact DFD on random, time-warped, zigzag and backtracking curves."""
import numpy as np
import pytest

import oracle


def anchors_and_inflation(X, k):
    n = len(X)
    idx = list(range(0, n - 1, k)) + [n - 1] if n > 1 else [0]
    idx = sorted(set(idx))
    cn = len(idx)
    infl = np.zeros(cn)

    def radius(b, tail):
        lo, hi = idx[b], idx[b + 1]
        mid = lo + (hi - lo) // 2
        pts = range(mid + 1, hi) if tail else range(lo + 1, min(mid, hi - 1) + 1)
        ref = X[hi] if tail else X[lo]
        return max([float(np.sqrt(np.sum((X[i] - ref) ** 2))) for i in pts], default=0.0)

    for a in range(cn):
        before = radius(a - 1, True) if a > 0 else 0.0
        after = radius(a, False) if a + 1 < cn else 0.0
        infl[a] = max(before, after)
    return X[idx], infl


def inflated_dfd(P, Q, k):
    A, ia = anchors_and_inflation(P, k)
    B, ib = anchors_and_inflation(Q, k)
    W = (np.sqrt(((A[:, None, :] - B[None, :, :]) ** 2).sum(-1)) + ia[:, None] + ib[None, :]) ** 2
    D = np.empty_like(W)
    for i in range(len(A)):
        for j in range(len(B)):
            if i == 0 and j == 0:
                best = -np.inf
            elif i == 0:
                best = D[0, j - 1]
            elif j == 0:
                best = D[i - 1, 0]
            else:
                best = min(D[i - 1, j], D[i, j - 1], D[i - 1, j - 1])
            D[i, j] = max(W[i, j], best)
    return float(np.sqrt(D[-1, -1]))


def curves(seed):
    rng = np.random.default_rng(seed)
    d = 2 + seed % 2
    kind = seed % 4
    n1, n2 = (int(v) for v in rng.integers(5, 90, 2))
    if kind == 0:  # random walks
        return np.cumsum(rng.normal(size=(n1, d)), 0), np.cumsum(rng.normal(size=(n2, d)), 0)
    if kind == 1:  # one path sampled twice, at uneven rates (dense and sparse stretches)
        t = np.sort(rng.random(200))
        path = np.cumsum(rng.normal(size=(200, d)), 0)
        s1 = np.sort(rng.random(n1) ** 3)
        s2 = np.sort(1 - rng.random(n2) ** 3)
        f = lambda s: np.stack([np.interp(s, t, path[:, e]) for e in range(d)], 1)
        return f(s1), f(s2) + rng.normal(scale=0.05, size=(n2, d))
    if kind == 2:  # zigzags of different periods
        x1, x2 = np.linspace(0, 10, n1), np.linspace(0, 10, n2)
        P = np.stack([x1, np.sign(np.sin(3 * x1))] + [x1 * 0] * (d - 2), 1)
        Q = np.stack([x2, np.sin(2 * x2)] + [x2 * 0] * (d - 2), 1)
        return P, Q
    # backtracking along a line against a straight curve
    P = np.zeros((n1, d))
    P[:, 0] = np.cumsum(rng.choice([1.0, 1.0, -0.7], size=n1))
    Q = np.zeros((n2, d))
    Q[:, 0] = np.linspace(P[0, 0], P[-1, 0], n2)
    return P, Q


@pytest.mark.parametrize("k", [2, 3, 4, 8, 17])
def test_inflated_anchor_dfd_bounds_the_dfd(k):
    for seed in range(24):
        P, Q = curves(seed)
        exact = float(np.sqrt(oracle.dfd_sq(P, Q)))
        bound = inflated_dfd(P, Q, k)
        assert bound * (1 + 2.0 ** -40) >= exact, (seed, k, bound, exact)


def test_every_point_an_anchor_is_the_dfd():
    for seed in range(8):
        P, Q = curves(seed)
        exact = float(np.sqrt(oracle.dfd_sq(P, Q)))
        assert abs(inflated_dfd(P, Q, 1) - exact) <= 1e-12 * max(1.0, exact)
