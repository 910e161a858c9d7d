"""The CPU oracle against known answers (no GPU).

The reference ships no tests or golden data; these pin the oracle with mathematical
known-answer cases, with its own sequential/parallel consistency and (test_golden.py)
with outputs of the reference's GPU code run on the same inputs.
"""
import math

import numpy as np
import pytest

import oracle


def line(n, y=0.0, x0=0.0, x1=1.0):
    return np.stack([np.linspace(x0, x1, n), np.full(n, y)], 1)


def test_parallel_lines():
    P = np.array([[0, 0], [1, 0], [2, 0]], float)
    Q = np.array([[0, 1], [2, 1]], float)
    assert oracle.endpoint(P, Q) == 1.0
    assert math.sqrt(oracle.dfd_sq(P, Q)) == math.sqrt(2.0)
    assert math.sqrt(oracle.vefd_sq(P, Q, 1.0)) == 1.0
    assert oracle.decide(P, Q, 1.0 + 1e-9)[0]
    assert not oracle.decide(P, Q, 1.0 - 1e-9)[0]
    r = oracle.distance(P, Q, stop_mode=1, quirks=False)
    assert abs(r["distance"] - 1.0) < 1e-9


def test_identical_curves_zero():
    rng = np.random.default_rng(1)
    P = np.cumsum(rng.normal(size=(50, 3)), 0)
    assert oracle.dfd_sq(P, P) == 0.0
    r = oracle.distance(P, P, stop_mode=1, quirks=False)
    # The VE-FD's projection parameter is a dot product over a squared length, the two
    # summed in different fused orders (as the reference's kernel compiles), so it can land a
    # rounding below 1 and leave a weight of a few ulps: lb may sit just above ub = 0.
    assert r["dfd"] == 0.0 and r["probes"] == 0
    assert 0.0 <= r["distance"] <= 1e-15


def test_single_segments_max_endpoint():
    P = np.array([[0.0, 0.0], [4.0, 1.0]])
    Q = np.array([[0.5, 2.0], [3.0, -1.0]])
    want = max(np.linalg.norm(P[0] - Q[0]), np.linalg.norm(P[1] - Q[1]))
    r = oracle.distance(P, Q, stop_mode=1, quirks=False)
    assert abs(r["distance"] - want) <= 1e-9 * want


@pytest.mark.parametrize("v", [(0.0, 0.7), (0.3, -0.4), (2.0, 1.0)])
def test_translated_straight_line(v):
    P = line(40, 0.0, 0.0, 10.0)
    Q = line(25, 0.0, 0.0, 10.0) + np.array(v)
    want = math.hypot(*v)
    r = oracle.distance(P, Q, stop_mode=1, quirks=False)
    assert abs(r["distance"] - want) <= 2e-9 * max(want, 1.0)


def walk_pair(seed, n1, n2, d=2, noise=0.05):
    rng = np.random.default_rng(seed)
    P = np.cumsum(rng.normal(size=(n1, d)), 0)
    idx = np.linspace(0, n1 - 1, n2)
    base = np.stack([np.interp(idx, np.arange(n1), P[:, k]) for k in range(d)], 1)
    return P, base + rng.normal(scale=noise, size=(n2, d))


@pytest.mark.parametrize("seed,d", [(0, 2), (1, 3), (2, 2), (3, 3)])
def test_bound_ordering_and_monotone_decisions(seed, d):
    P, Q = walk_pair(seed, 60, 45, d)
    r = oracle.distance(P, Q, stop_mode=1, quirks=False)
    fd = r["distance"]
    assert r["endpoint"] <= r["vefd"] * (1 + 1e-12)
    assert r["vefd"] <= fd * (1 + 1e-9)
    assert fd <= r["dfd"] * (1 + 1e-9)
    grid = np.linspace(r["vefd"] * 0.9, r["dfd"] * 1.1, 41)
    dec = [oracle.decide(P, Q, e)[0] for e in grid]
    assert dec == sorted(dec)  # False...False True...True
    assert oracle.decide(P, Q, fd * (1 + 1e-8))[0]
    assert not oracle.decide(P, Q, fd * (1 - 1e-8))[0]


@pytest.mark.parametrize("n1,n2", [(3, 200), (300, 7), (130, 1100), (1500, 90)])
def test_parallel_sweep_bitexact(n1, n2):
    """The anti-diagonal tile sweep equals the sequential sweep bit for bit."""
    P, Q = walk_pair(n1 + n2, n1, n2, 3)
    assert oracle.dfd_sq(P, Q, 1) == oracle.dfd_sq(P, Q, 8)
    lb = oracle.endpoint(P, Q)
    assert oracle.vefd_sq(P, Q, lb, 1) == oracle.vefd_sq(P, Q, lb, 8)
    for e in (0.5, 1.0, 2.0, 4.0):
        assert oracle.decide(P, Q, e, 1)[1] == oracle.decide(P, Q, e, 8)[1]


def brute_dfd(P, Q):
    n, m = len(P), len(Q)
    D = np.full((n, m), np.inf)
    for i in range(n):
        for j in range(m):
            d = float(np.sum((P[i] - Q[j]) ** 2))
            if i == 0 and j == 0:
                D[i, j] = d
            else:
                best = min(D[i - 1, j] if i else np.inf, D[i, j - 1] if j else np.inf,
                           D[i - 1, j - 1] if i and j else np.inf)
                D[i, j] = max(d, best)
    return D[-1, -1]


@pytest.mark.parametrize("seed", range(4))
def test_dfd_matches_textbook_recurrence(seed):
    """The reference's folded DFD (min passed down includes the diagonal) equals the
    textbook three-predecessor recurrence."""
    P, Q = walk_pair(seed + 10, 17, 23, 2)
    assert abs(oracle.dfd_sq(P, Q) - brute_dfd(P, Q)) <= 1e-12 * brute_dfd(P, Q)


def brute_vefd(P, Q, lb):
    """Bottleneck path over vertex-edge events (README.md:77-126 of the reference)."""
    def seg(x, a, b):
        ab = b - a
        t = min(1.0, max(0.0, float(np.dot(x - a, ab) / np.dot(ab, ab))))
        return float(np.sum((x - (a + t * ab)) ** 2))
    m, n = len(P) - 1, len(Q) - 1
    T = np.full((m, n), np.inf)
    R = np.full((m, n), np.inf)
    for i in range(m):
        for j in range(n):
            below = T[i, j - 1] if j else (lb * lb if i == 0 else np.inf)
            left = R[i - 1, j] if i else np.inf
            inc = min(below, left)
            T[i, j] = max(seg(Q[j + 1], P[i], P[i + 1]), inc)
            R[i, j] = max(seg(P[i + 1], Q[j], Q[j + 1]), inc)
    return min(T[-1, -1], R[-1, -1])


@pytest.mark.parametrize("seed", range(4))
def test_vefd_matches_bottleneck_definition(seed):
    P, Q = walk_pair(seed + 20, 14, 19, 3)
    lb = oracle.endpoint(P, Q)
    want = brute_vefd(P, Q, lb)
    assert abs(oracle.vefd_sq(P, Q, lb) - want) <= 1e-12 * want


def test_reference_stop_rule_and_quirk():
    P, Q = walk_pair(7, 60, 50, 2)  # 60*50 <= 10000: the reference skips VE-FD
    r = oracle.distance(P, Q, stop_mode=0, quirks=True)
    assert r["vefd"] == r["endpoint"]
    assert r["ub"] - r["lb"] <= oracle.FLT_EPSILON
    assert r["distance"] == (r["ub"] + r["lb"]) / 2
    r2 = oracle.distance(P, Q, stop_mode=0, quirks=False)
    assert r2["vefd"] >= r["vefd"]
    assert abs(r2["distance"] - r["distance"]) <= oracle.FLT_EPSILON


def test_materialised_formula_rounds_differently():
    """The reference's two decision paths round C of the quadratic differently: the
    materialised path forms (sum mi^2) - r^2 (src/intersection_algorithm_in_parallel.cu:742),
    the fused one sums from -r^2 (.cu:1177-1186).  Their intervals differ in the last bits for
    some partial edges, never by more than a few ulps of the edge parameter, and agree on
    emptiness away from tangency."""
    rng = np.random.default_rng(7)
    n = 50000
    X = rng.normal(size=(n, 3)) * 100.0
    a = X + rng.normal(size=(n, 3))
    b = a + rng.normal(size=(n, 3))
    A = ((b - a) ** 2).sum(1)
    r2 = float(np.median(((a - X) ** 2).sum(1)))
    l0, h0 = oracle.free_intervals(X, a, b, A, r2)
    l1, h1 = oracle.free_intervals(X, a, b, A, r2, formula=1)
    part = (l0 >= 0) & (l1 >= 0)
    assert (l0 != l1).sum() + (h0 != h1).sum() > 100
    assert np.max(np.abs(l0[part] - l1[part])) < 1e-9
    assert np.max(np.abs(h0[part] - h1[part])) < 1e-9
    assert ((l0 < 0) != (l1 < 0)).sum() < 5


def test_materialised_search_close_to_fused():
    P, Q = oracle.gen_pair(1, 3, 400, 350, 100.0, 0.1, 8, 0)
    a = oracle.distance(P, Q, stop_mode=1, quirks=False)
    b = oracle.distance(P, Q, stop_mode=1, quirks=False, formula=1)
    assert abs(a["distance"] - b["distance"]) <= 2.0 ** -32 * a["distance"]
    assert a["vefd"] == b["vefd"] and a["dfd"] == b["dfd"]
